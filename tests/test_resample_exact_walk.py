"""The float arithmetic behind resample's exact walk (rpp_b200/csrc/resample.cu, resample_exact_range).

The reference computes every tap of an output at phase p with float operations
(src/modules/tensor/cpu/kernel/resample.cpp:83-115, api/rppdefs.h:760-782):
- the offset x = l - p, then lanes x + 1, x + 2, x + 3, each stepped by 4;
- the table position x * scale + center;
- its floor, and the weight position - floor.

For scale 32, an integer center, and p at or above 2^Emin (Emin from lobes and center, as in
resample_exact_range), the claim is that none of these operations rounds. Consecutive taps then sit
exactly 32 table entries apart and share one weight. The GPU kernel relies on this to read each tap's
entry 32 entries past the previous one. This test replays the reference's per-tap float operations in
numpy on random phases and checks the claim. It also checks that below Emin the claim fails for some
phases, so the threshold is not loose by a binade.
"""
import numpy as np
import pytest

F32 = np.float32


def exact_min_exponent(lobes, center):
    """The smallest E for which phases in [2^E, 2^19) take the exact walk (resample_exact_range)."""
    for e in range(-126, 19):
        if lobes < 2.0 ** (e + 1) and center + 32.0 * lobes < 2.0 ** (e + 6):
            return e
    return None


def tap_positions(p, lobes, center, shift):
    """Per tap t: (floor of the table position, weight) by the reference's float operations.
    shift > 0 starts the taps later, as at a signal's start."""
    loc0 = np.ceil(p.astype(np.float64)).astype(np.int64) - lobes + shift
    loc1 = np.ceil(p.astype(np.float64)).astype(np.int64) + lobes
    ntap = int((loc1 - loc0).min())
    locBegin = (loc0.astype(F32) - p).astype(F32)
    lanes = [(locBegin + F32(j)).astype(F32) for j in range(4)]

    def pos(x):   # fmaf(x, 32, center): exact in float64, one rounding to float
        r = (x.astype(np.float64) * 32.0 + center).astype(F32)
        m = np.floor(r.astype(np.float64))
        return m, (r - m.astype(F32)).astype(F32)

    out = []
    groups = ntap // 4
    for _ in range(groups):
        for j in range(4):
            out.append(pos(lanes[j]))
            lanes[j] = (lanes[j] + F32(4)).astype(F32)
    xx = ((loc0 + 4 * groups).astype(F32) - p).astype(F32)
    for _ in range(4 * groups, ntap):
        out.append(pos(xx))
        xx = (xx + F32(1)).astype(F32)
    return out


def walk_holds(p, lobes, center, shift):
    taps = tap_positions(p, lobes, center, shift)
    m0, w0 = taps[0]
    ok = np.ones(p.shape, bool)
    for t, (m, w) in enumerate(taps):
        ok &= (m == m0 + 32 * t) & (w.view(np.uint32) == w0.view(np.uint32))
    return ok


@pytest.mark.parametrize("lobes", [8, 16, 24])
def test_exact_walk_holds_from_the_threshold(lobes):
    center = float(lobes * 32 + 1)   # windowed_sinc's center for lobes * 64 + 1 coefficients
    emin = exact_min_exponent(lobes, center)
    assert emin is not None
    r = np.random.default_rng(lobes)
    for e in range(emin, 19):
        p = (r.uniform(1.0, 2.0, 4000) * 2.0 ** e).astype(F32)
        for shift in (0, 3):
            assert walk_holds(p, lobes, center, shift).all(), (lobes, e, shift)
    # one binade lower, some phases break it
    p = (r.uniform(1.0, 2.0, 4000) * 2.0 ** (emin - 1)).astype(F32)
    assert not walk_holds(p, lobes, center, 0).all()
