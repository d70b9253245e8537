"""Builds rpp_b200/librppb.so (the C-ABI library of the audio path) with nvcc for sm_100a.

Each rpp_b200/csrc/*.cu file is compiled to an object in rpp_b200/_build/ (in parallel, only when
it or a header changed) and linked into an in-tree shared library with the CUDA runtime linked
statically, so the library loads next to any PyTorch/CUDA runtime in the process.

--checked builds rpp_b200/librppb_checked.so instead (objects in rpp_b200/_build_checked/): the same
sources with -DRPPB_CHECKED and relocatable device code, in which every global access of the kernels
is checked against the regions of the call that launched it (rpp_b200/csrc/check.cu).  Load it with
RPPB_LIBRARY=checked (rpp_b200/lib.py).

    python -m rpp_b200.build [--verbose-ptxas] [--checked]
"""
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "librppb.so")
OBJ_CHECKED = os.path.join(HERE, "_build_checked")
LIB_CHECKED = os.path.join(HERE, "librppb_checked.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.isfile(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def _flags(ptxas_verbose=False, checked=False):
    f = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "--expt-relaxed-constexpr"]
    if checked:
        f += ["-DRPPB_CHECKED", "-rdc=true"]
    if ptxas_verbose:
        f += ["-Xptxas", "-v"]
    return f


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def build(force=False, ptxas_verbose=False, jobs=None, checked=False):
    objdir, lib = (OBJ_CHECKED, LIB_CHECKED) if checked else (OBJ, LIB)
    os.makedirs(objdir, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr = _newest_header()
    cc = nvcc()
    flags = _flags(ptxas_verbose, checked)

    def one(src):
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        if not force and os.path.isfile(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr):
            return obj, ""
        # the checked build's access check is called from kernels launched with as few as 32 registers
        extra = ["-maxrregcount=32"] if checked and os.path.basename(src) == "check.cu" else []
        r = subprocess.run([cc] + flags + extra + ["-c", src, "-o", obj], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
        return obj, r.stderr

    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(one, srcs))
    objs = [o for o, _ in results]
    logs = "".join(l for _, l in results)
    if force or not os.path.isfile(lib) or os.path.getmtime(lib) < max(os.path.getmtime(o) for o in objs):
        link = ["-rdc=true"] if checked else []
        r = subprocess.run([cc] + ARCH + link + ["-shared", "-cudart", "static", "-o", lib + ".tmp"] + objs,
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
        os.replace(lib + ".tmp", lib)
    return lib, logs


if __name__ == "__main__":
    v = "--verbose-ptxas" in sys.argv
    lib, logs = build(force="--force" in sys.argv or v, ptxas_verbose=v, checked="--checked" in sys.argv)
    if v:
        print(logs)
    print(lib)
