"""Helpers for the GPU tests: torch CUDA tensors as device memory, pinned host tensors for
per-sample arguments, and the comparison metrics with their tolerances."""
import numpy as np
import torch


def dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def pinned(a):
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def canvas(shape, fill=-12345.0):
    """Output buffer pre-filled with a canary value, to check that nothing outside the valid
    region is written."""
    return torch.full(shape, fill, dtype=torch.float32, device="cuda")


# Parity bounds (per-frame relative for spectra; absolute dB).
SPEC_FRAME_REL = 1e-5
DB_ABS = 1e-3


def frame_rel_err(got, ref, axis=0):
    """max |got - ref| / max(ref along `axis`) over all frames (power spectra, mel)."""
    ref = np.asarray(ref, np.float64)
    scale = np.maximum(np.abs(ref).max(axis=axis, keepdims=True), 1e-30)
    return float((np.abs(np.asarray(got, np.float64) - ref) / scale).max()) if ref.size else 0.0
