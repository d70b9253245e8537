"""Resampling-window lookup tables in the layout RpptResamplingWindow expects
(api/rppdefs.h:751-790): lut[0] = 0, lut[i + 1] = w((i - center0) / (coeffs - 1) * 2 * lobes) for
i < coeffs, four trailing zeros; the window reads lut at x * scale + center for an input sample x
periods away from the output position, with scale = (coeffs - 1) / (2 * lobes) and
center = center0 + 1.  Weights are evaluated in FP64 and rounded once to float.
"""
import numpy as np


def kaiser_sinc(lobes=16, coeffs=None, beta=8.0):
    """Kaiser-windowed sinc with `lobes` zero crossings on each side (beta stated by the caller;
    8.0 gives ~ -80 dB side lobes).  Returns (lut float32, scale, center, lobes)."""
    coeffs = coeffs or lobes * 64 + 1
    center0 = (coeffs - 1) // 2
    i = np.arange(coeffs, dtype=np.float64)
    x = (i - center0) * (2.0 * lobes / (coeffs - 1))           # in input periods, [-lobes, lobes]
    t = (i - center0) / center0                                 # [-1, 1] across the table
    env = np.i0(beta * np.sqrt(np.clip(1.0 - t * t, 0.0, 1.0))) / np.i0(beta)
    lut = np.zeros(coeffs + 5, np.float64)
    lut[1:coeffs + 1] = np.sinc(x) * env
    return lut.astype(np.float32), float(np.float32((coeffs - 1) / (2.0 * lobes))), float(center0 + 1), int(lobes)
