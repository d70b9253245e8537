"""Runs every entry point of the audio path once on the 256-clip batch (ragged 16 kHz clips,
1-16 s) and the first 256 clips of the stereo multi-rate batch (mixed rates), for kernel profiling:

    python -m rpp_b200.profile_ops [--clips N] [--repeat R]

With --repeat 1 (the default) each kernel of the path launches once per entry point (plus the small
ragged-prefix kernels), so `ncu -k regex:... -c <count>` captures each kernel once.  The inputs
are larger than L2.  Prints one line per entry point with its CUDA-event time of the last repeat.
"""
import argparse
import ctypes

import numpy as np
import torch

from . import audio, lib, synth
from .types import audio_desc, spectra_desc, frontend_params, generic_desc
from .windows import kaiser_sinc


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--clips", type=int, default=256)
    ap.add_argument("--repeat", type=int, default=1)
    args = ap.parse_args()
    L_ = lib.load()
    dev = torch.device("cuda")
    h = lib.Handle(batch_size=args.clips, stream=torch.cuda.current_stream().cuda_stream)
    x_np, lens_np = synth.gapped_clips(n=args.clips)
    n, L = x_np.shape
    x = torch.from_numpy(x_np).to(dev)
    lens = torch.from_numpy(lens_np).to(dev)
    coeff = torch.full((n,), 0.97, device=dev)
    F = (lens_np // 160 + 1).astype(np.int32)
    mf = int(F.max())
    sd = audio_desc(n, L)
    spd, md = spectra_desc(n, 257, mf), spectra_desc(n, 128, mf)
    pre = torch.empty_like(x)
    spec = torch.empty((n, 257, mf), device=dev)
    mel = torch.empty((n, 128, mf), device=dev)
    db = torch.empty_like(mel)
    dims = torch.from_numpy(np.stack([np.full(n, 257, np.int32), F], 1).astype(np.int32)).to(dev)
    patches = torch.from_numpy(np.stack([F, np.full(n, 128, np.int32)], 1).astype(np.int32)).to(dev)
    begin = torch.empty(n, dtype=torch.int32, device=dev)
    length = torch.empty(n, dtype=torch.int32, device=dev)
    p = frontend_params()

    # stereo multi-rate subset
    xs_np, ls_np, rates_np = synth.stereo_multirate_clips(n=args.clips)
    Ls = int(ls_np.max())
    xs = torch.from_numpy(xs_np).to(dev)
    sdims = torch.from_numpy(np.stack([ls_np, np.full(args.clips, 2, np.int32)], 1).astype(np.int32)).to(dev)
    mono = torch.empty((args.clips, Ls), device=dev)
    lut, scale, center, lobes = kaiser_sinc(16, beta=8.0)
    lut_d = torch.from_numpy(lut).to(dev)
    win = audio.resampling_window(lut_d, scale, center, lobes)
    ir = torch.from_numpy(rates_np).to(dev)
    orr = torch.full((args.clips,), 16000.0, device=dev)
    L16 = int(np.ceil(Ls * 16000.0 / float(rates_np.min()))) + 8
    mono16 = torch.empty((args.clips, L16), device=dev)
    mdims = torch.from_numpy(np.stack([ls_np, np.ones(args.clips, np.int32)], 1).astype(np.int32)).to(dev)

    x_host = torch.from_numpy(x_np).pin_memory()
    out_host = torch.empty((n, 128, mf)).pin_memory()
    lens_host = torch.from_numpy(lens_np).pin_memory()
    coeff_host = torch.full((n,), 0.97).pin_memory()
    db_small = torch.empty((min(n, 8), 128, mf), device=dev)
    dims_small = patches[:min(n, 8)].contiguous()
    sd_small = spectra_desc(min(n, 8), 128, mf)
    stream = torch.cuda.current_stream().cuda_stream
    gd = generic_desc((n, L))
    sl_anchor = torch.full((n,), 10, dtype=torch.int32, device=dev)
    sl_shape = torch.from_numpy((lens_np // 2).astype(np.int32)).to(dev)
    sl_roi = torch.from_numpy(np.stack([np.full(n, 10), lens_np], 1).astype(np.uint32).ravel().view(np.int32)).to(dev)
    sl_fill = torch.zeros(1, device=dev)
    nd = generic_desc((n, 128, mf))
    n_roi = torch.from_numpy(np.stack([np.zeros(n), np.zeros(n), np.full(n, 128), F], 1).astype(np.uint32).ravel()
                             .view(np.int32))
    n_mean, n_std = torch.zeros(n * 128, device=dev), torch.zeros(n * 128, device=dev)
    n_out = torch.empty_like(db)

    ops = [
        ("pre_emphasis_filter", lambda: audio.pre_emphasis_filter(x, sd, pre, sd, lens, coeff, 0, h)),
        ("spectrogram", lambda: audio.spectrogram(pre, sd, spec, spd, lens, True, True, None, 512, 2, 400, 160, h)),
        ("mel_filter_bank", lambda: audio.mel_filter_bank(spec, spd, mel, md, dims, 8000.0, 0.0, 0, 128, 16000.0,
                                                          True, h)),
        ("to_decibels", lambda: audio.to_decibels(mel, md, db, md, patches, -80.0, 10.0, 0.0, h)),
        ("frontend (fused)", lambda: audio.frontend(x, sd, db, md, lens, coeff, p, h)),
        ("non_silent_region_detection", lambda: audio.non_silent_region_detection(x, sd, lens, begin, length, -60.0,
                                                                                  2048, 0.0, 8192, h)),
        ("down_mixing", lambda: audio.down_mixing(xs, audio_desc(args.clips, Ls, channels=2, num_dims=3), mono,
                                                  audio_desc(args.clips, Ls), sdims, False, h)),
        ("resample", lambda: audio.resample(mono, audio_desc(args.clips, Ls), mono16, audio_desc(args.clips, L16), ir,
                                            orr, mdims, win, h)),
        ("downmix_resample (fused)", lambda: audio.downmix_resample(xs, audio_desc(args.clips, Ls, channels=2,
                                                                                   num_dims=3),
                                                                    mono16, audio_desc(args.clips, L16), ir, orr,
                                                                    sdims, False, lut_d, scale, center, lobes, h)),
        ("spectrogram_tc (BF16 hi/lo x3)", lambda: audio.spectrogram_tc(x, sd, spec, spd, lens, coeff, 0, True, True,
                                                                         512, 2, 400, 160, audio.TC_BF16_HILO3, h)),
        ("frontend_host (pinned host tensors)", lambda: audio.frontend_host(x_host, sd, out_host, md, lens_host,
                                                                            coeff_host, p, 0, h)),
        ("slice (1-D, anchor 10, length/2)", lambda: audio.slice(x, gd, pre, gd, sl_anchor, sl_shape, sl_fill, True,
                                                                 sl_roi, h)),
        ("normalize (per filter over time)", lambda: audio.normalize(db, nd, n_out, nd, 2, n_mean, n_std, 3, 1.0, 0.0,
                                                                     n_roi, h)),
        ("to_decibels_gpu_static (8 clips)", lambda: L_.rppt_to_decibels_gpu_static(
            mel.data_ptr(), ctypes.byref(sd_small), db_small.data_ptr(), ctypes.byref(sd_small),
            dims_small.data_ptr(), ctypes.c_float(-80.0), ctypes.c_float(10.0), ctypes.c_float(0.0),
            ctypes.c_void_p(stream))),
    ]
    for name, fn in ops:
        for _ in range(args.repeat):
            st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            st.record()
            rc = fn()
            en.record()
            torch.cuda.synchronize()
            if rc != 0:
                raise RuntimeError(f"{name}: status {rc} {lib.last_error()}")
        print(f"{name:40s} {st.elapsed_time(en):9.3f} ms")
    assert audio.device_error(h) == 0
    h.close()


if __name__ == "__main__":
    main()
