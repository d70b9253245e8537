"""The C-ABI boundary without a GPU: the library loads, exports every symbol the public headers
declare, and the headers keep the reference's type layouts and enum values."""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from rpp_b200 import lib
from rpp_b200 import types as T

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
REF = os.environ.get("RPP_REF", os.path.join(os.path.dirname(ROOT), "reference"))


def declared_symbols():
    names = set()
    for h in os.listdir(INCLUDE):
        if h.endswith(".h"):
            text = open(os.path.join(INCLUDE, h)).read()
            names |= set(re.findall(r"SHARED_PUBLIC\s+[\w\s\*]+?\b(\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    L = lib.load()
    declared = declared_symbols()
    assert {"rppCreate", "rppt_spectrogram_gpu", "rppt_resample_gpu"} <= declared
    for name in sorted(declared | set(lib.EXPORTED)):
        assert hasattr(L, name), name


def test_no_host_backend():
    h = ctypes.c_void_p()
    st = lib.load().rppCreate(ctypes.byref(h), 1, 0, None, int(T.RppBackend.RPP_HOST_BACKEND))
    assert st == T.RppHandleStatus.rppStatusNotImplemented


def test_create_without_device_fails_cleanly():
    """With no usable GPU rppCreate returns an error status instead of aborting."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    st = lib.load().rppCreate(ctypes.byref(h), 1, 0, None, int(T.RppBackend.RPP_HIP_BACKEND))
    assert st != 0


def test_null_handle_status():
    d = T.audio_desc(1, 16)
    st = lib.load().rppt_pre_emphasis_filter_gpu(None, ctypes.byref(d), None, ctypes.byref(d), None, None, 0, None)
    assert st == T.RppStatus.RPP_ERROR_INVALID_ARGUMENTS


LAYOUT_PROBE = r"""
#include <cstdio>
#include <cstddef>
#include "rppdefs.h"
int main() {
  std::printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(RpptDesc), offsetof(RpptDesc, strides), offsetof(RpptDesc, layout),
              sizeof(RpptImagePatch), sizeof(RpptResamplingWindow), offsetof(RpptResamplingWindow, lookup),
              offsetof(RpptResamplingWindow, pCenter));
  std::printf("%zu %zu %zu %zu\n", sizeof(RpptGenericDesc), offsetof(RpptGenericDesc, dims),
              offsetof(RpptGenericDesc, strides), offsetof(RpptGenericDesc, layout));
  std::printf("%d %d %d %d %d %d %d %d\n", (int)RPP_ERROR_INVALID_AXIS, (int)RPP_ERROR_OUT_OF_BOUND_SCRATCH_MEMORY_SIZE,
              (int)NFT, (int)NTF, (int)REFLECT, (int)HTK, (int)F32, (int)RPP_HIP_BACKEND);
  return 0;
}
"""


def _probe(include_dirs, extra=()):
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "p.cpp")
        exe = os.path.join(d, "p")
        open(src, "w").write(LAYOUT_PROBE)
        cmd = ["g++", "-std=c++17", "-w", src, "-o", exe] + [f"-I{i}" for i in include_dirs] + list(extra)
        subprocess.run(cmd, check=True, capture_output=True)
        return subprocess.run([exe], check=True, capture_output=True, text=True).stdout


def test_header_layout_matches_ctypes():
    out = _probe([INCLUDE]).split("\n")
    sizes = [int(v) for v in out[0].split()]
    assert sizes[0] == ctypes.sizeof(T.RpptDesc)
    assert sizes[1] == T.RpptDesc.strides.offset
    assert sizes[2] == T.RpptDesc.layout.offset
    assert sizes[3] == ctypes.sizeof(T.RpptImagePatch)
    assert sizes[4] == ctypes.sizeof(T.RpptResamplingWindow)
    assert sizes[5] == T.RpptResamplingWindow.lookup.offset
    assert sizes[6] == T.RpptResamplingWindow.pCenter.offset
    g = [int(v) for v in out[1].split()]
    assert g == [ctypes.sizeof(T.RpptGenericDesc), T.RpptGenericDesc.dims.offset, T.RpptGenericDesc.strides.offset,
                 T.RpptGenericDesc.layout.offset]


def test_header_layout_matches_reference():
    """Same probe compiled against the reference's api/rppdefs.h (where the sources exist)."""
    if not os.path.isdir(os.path.join(REF, "api")):
        pytest.skip("reference headers absent")
    gen = os.path.join(ROOT, "oracle", "_ref", "gen")
    if not os.path.isdir(gen):
        pytest.skip("oracle/_ref/gen missing (run oracle/build_ref.sh)")
    ours = _probe([INCLUDE])
    theirs = _probe([gen, os.path.join(REF, "api")], extra=["-mavx2", "-mf16c"])
    assert ours == theirs


def test_headers_compile_as_c():
    """Every public header compiles in a C translation unit (gnu11, as gcc builds C by default), so
    C callers and FFI bindings generated from the headers can include them; the C++-only
    RpptResamplingWindow is hidden from C by the headers themselves."""
    import shutil
    if shutil.which("gcc") is None:
        pytest.skip("gcc absent")
    headers = sorted(f for f in os.listdir(INCLUDE) if f.endswith(".h"))
    src = "".join(f'#include "{h}"\n' for h in headers) + "int main(void) { return sizeof(RpptDesc) == 0; }\n"
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "c_headers.c")
        open(path, "w").write(src)
        r = subprocess.run(["gcc", "-std=gnu11", "-Wall", "-Wextra", "-Werror", f"-I{INCLUDE}", "-fsyntax-only", path],
                           capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
