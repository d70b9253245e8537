"""Captures the reference's audio QA fixtures as compact .npz files under tests/golden/.

Run once in a checkout that has the reference sources (default ../reference beside this repository,
or $RPP_REF);
the GPU tests read only the .npz files this writes.  Sources of each array:
  inputs  utilities/test_suite/TEST_AUDIO_FILES/three_samples_single_channel_src1/sample{1,2,3}.wav
          (16 kHz mono int16; the test suite reads them with libsndfile's sf_read_float, i.e.
          int16 / 32768, utilities/test_suite/rpp_test_suite_audio.h:143-178)
  goldens utilities/test_suite/REFERENCE_OUTPUTS_AUDIO/<op>/<op>.bin (raw float32, laid out
          [3][nStride] with the test suite's strides, rpp_test_suite_audio.h:252-343)
  NSR     the {begin, length} triples of rpp_test_suite_audio.h:64-69
"""
import os
import sys
import wave

import numpy as np

REF = os.environ.get("RPP_REF", os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))), "reference"))
HERE = os.path.dirname(os.path.abspath(__file__))
SUITE = os.path.join(REF, "utilities", "test_suite")


def main():
    wavdir = os.path.join(SUITE, "TEST_AUDIO_FILES", "three_samples_single_channel_src1")
    pcm = []
    for i in (1, 2, 3):
        with wave.open(os.path.join(wavdir, f"sample{i}.wav")) as w:
            assert w.getnchannels() == 1 and w.getsampwidth() == 2 and w.getframerate() == 16000
            pcm.append(np.frombuffer(w.readframes(w.getnframes()), dtype="<i2").copy())
    lengths = np.array([len(p) for p in pcm], dtype=np.int32)
    out = {"lengths": lengths}
    for i, p in enumerate(pcm):
        out[f"pcm{i}"] = p
    gold = os.path.join(SUITE, "REFERENCE_OUTPUTS_AUDIO")
    for op in ("pre_emphasis_filter", "to_decibels", "spectrogram", "mel_filter_bank", "resample", "slice"):
        out[op] = np.fromfile(os.path.join(gold, op, op + ".bin"), dtype="<f4")
    out["nsr_begin"] = np.array([0, 0, 0], dtype=np.int32)
    out["nsr_length"] = np.array([35840, 33680, 34160], dtype=np.int32)
    dst = os.path.join(HERE, "reference_audio_qa.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, os.path.getsize(dst), "bytes")


if __name__ == "__main__":
    sys.exit(main())
