"""ORACLE — test infrastructure only.

Two CPU checkers for the GPU audio path, used by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product:

* ``Oracle``    — ctypes front of oracle/rppb_oracle.c, this repository's C restatement of the
                  reference's host audio path (float mirrors + FP64 forms);
* ``Reference`` — ctypes front of oracle/_ref/librpp_audio_ref.so, the reference's own host
                  (OpenMP) audio path compiled from its sources by oracle/build_ref.sh.
"""
from .oracle import Oracle, Reference, build_oracle, build_reference, oracle_lib_path, reference_lib_path  # noqa: F401
