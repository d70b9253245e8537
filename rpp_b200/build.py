"""Builds rpp_b200/librppb.so (the C-ABI library of the audio path) with nvcc for sm_100a.

Each rpp_b200/csrc/*.cu file is compiled to an object in rpp_b200/_build/ (in parallel, only when
it or a header changed) and linked into an in-tree shared library with the CUDA runtime linked
statically, so the library loads next to any PyTorch/CUDA runtime in the process.

    python -m rpp_b200.build [--verbose-ptxas]
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
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.isfile(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def _flags(ptxas_verbose=False):
    f = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "--expt-relaxed-constexpr"]
    if ptxas_verbose:
        f += ["-Xptxas", "-v"]
    return f


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def build(force=False, ptxas_verbose=False, jobs=None):
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr = _newest_header()
    cc = nvcc()
    flags = _flags(ptxas_verbose)

    def one(src):
        obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
        if not force and os.path.isfile(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr):
            return obj, ""
        r = subprocess.run([cc] + flags + ["-c", src, "-o", obj], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
        return obj, r.stderr

    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(one, srcs))
    objs = [o for o, _ in results]
    logs = "".join(l for _, l in results)
    if force or not os.path.isfile(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        r = subprocess.run([cc] + ARCH + ["-shared", "-cudart", "static", "-o", LIB + ".tmp"] + objs,
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
        os.replace(LIB + ".tmp", LIB)
    return LIB, logs


if __name__ == "__main__":
    v = "--verbose-ptxas" in sys.argv
    lib, logs = build(force="--force" in sys.argv or v, ptxas_verbose=v)
    if v:
        print(logs)
    print(lib)
