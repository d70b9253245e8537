"""The continuous-batching server (native scheduler of include/rppb_server.h, driven through
rpp_b200/serving.py): each request's result is the same alone and in a mix of concurrently admitted
requests, under memory pressure, with pinned or pageable host buffers (copy kernels or DMA copies),
through the fused or the plain four-call step, and equals the descriptor-based calls
(rppb_downmix_resample_gpu + rppb_frontend_gpu) on the same clip."""
import numpy as np
import pytest
import torch

from rpp_b200 import audio, serving
from rpp_b200.types import RppStatus, audio_desc, spectra_desc, frontend_params
from rpp_b200.windows import kaiser_sinc

pytestmark = pytest.mark.gpu


def requests(seed, n):
    rng = np.random.Generator(np.random.PCG64(seed))
    return [serving.make_request(torch, i, rng, max_s=6.0) for i in range(n)]


def run(server, reqs, arrivals=None):
    for r in reqs:
        serving.attach_outputs(torch, server, r)
    done = server.run(reqs, arrivals)
    torch.cuda.synchronize()
    return {r.rid: [o.clone() for o in r.outputs] for r in done}


def test_alone_equals_mixed():
    server = serving.FrontendServer(torch, budget_bytes=1 << 30, max_clips=64, tables=3)
    mix = requests(7, 24)
    probe = mix[5]
    alone = run(server, [probe])[probe.rid]
    arrivals = list(np.linspace(0.0, 0.02, len(mix)))
    mixed = run(server, mix, arrivals)
    assert len(mixed) == len(mix)
    for a, b in zip(alone, mixed[probe.rid]):
        assert torch.equal(a, b)
    assert server.arena_used() == 0
    server.close()


def test_server_equals_descriptor_calls(gpu):
    server = serving.FrontendServer(torch, budget_bytes=1 << 28, max_clips=16, tables=2)
    reqs = requests(11, 3)
    out = run(server, reqs)
    lut, scale, center, lobes = kaiser_sinc(16)
    lut_d = torch.from_numpy(lut).cuda()
    p = frontend_params()
    for r in reqs:
        for c, rate, got in zip(r.clips, r.rates, out[r.rid]):
            L = c.numel()
            x = c.cuda().view(1, L)
            lr, f = server._frames(L, rate)
            mono = torch.zeros((1, lr + 8), device="cuda")
            dims = torch.tensor([[L, 1]], dtype=torch.int32, device="cuda")
            assert audio.downmix_resample(x, audio_desc(1, L), mono, audio_desc(1, lr + 8),
                                          torch.tensor([rate], device="cuda"), torch.tensor([16000.0], device="cuda"),
                                          dims, False, lut_d, scale, center, lobes, gpu) == RppStatus.RPP_SUCCESS
            dst = torch.full((1, 128, max(f, 1)), -7.0, device="cuda")
            assert audio.frontend(mono, audio_desc(1, lr + 8), dst, spectra_desc(1, 128, max(f, 1)),
                                  torch.tensor([lr], dtype=torch.int32, device="cuda"),
                                  torch.tensor([0.97], device="cuda"), p, gpu) == RppStatus.RPP_SUCCESS
            torch.cuda.synchronize()
            assert torch.equal(dst[0].cpu(), got)
    server.close()


def test_budget_pressure_and_oversize():
    """A budget that holds only a few requests at a time: FIFO admission waits for memory, every
    request completes with the same bits as on a large budget, the arena drains; a request that can
    never fit is refused at submission."""
    reqs = requests(23, 40)
    big = serving.FrontendServer(torch, budget_bytes=1 << 30, max_clips=64, tables=3)
    ref = run(big, reqs)
    big.close()
    small = serving.FrontendServer(torch, budget_bytes=24 << 20, max_clips=64, tables=3)
    got = run(small, reqs)
    assert len(got) == len(reqs)
    for r in reqs:
        for a, b in zip(ref[r.rid], got[r.rid]):
            assert torch.equal(a, b)
    assert small.arena_used() == 0
    huge = serving.Request(rid=999, clips=[torch.zeros(8 << 20).pin_memory()], rates=[16000.0], arrival=0.0)
    serving.attach_outputs(torch, small, huge)
    with pytest.raises(RuntimeError):
        small.submit(huge)
    small.close()


def test_plain_step_equals_fused_step():
    """The plain FP32 path (resample, then the four rppt_*_gpu calls on a batch buffer) gives the fused
    server's bits: the fused front end equals the four calls, and both read the same resampled clips."""
    reqs = requests(31, 16)
    fused = serving.FrontendServer(torch, budget_bytes=1 << 30, max_clips=32, tables=2)
    ref = run(fused, reqs)
    fused.close()
    plain = serving.FrontendServer(torch, budget_bytes=1 << 30, max_clips=32, tables=2, plain=True,
                                   max_samples=6 * 16000 + 16)
    got = run(plain, reqs, list(np.linspace(0.0, 0.01, len(reqs))))
    assert len(got) == len(reqs)
    for r in reqs:
        for a, b in zip(ref[r.rid], got[r.rid]):
            assert torch.equal(a, b)
    assert plain.arena_used() == 0
    # a clip longer than the plain path's batch rows is refused at submission
    long = serving.Request(rid=998, clips=[torch.zeros(7 * 16000).pin_memory()], rates=[16000.0], arrival=0.0)
    serving.attach_outputs(torch, plain, long)
    with pytest.raises(RuntimeError):
        plain.submit(long)
    plain.close()


def test_pageable_buffers_equal_pinned():
    """Clips and outputs in pageable host memory go through DMA copies instead of the copy kernels; the
    bits are the same."""
    reqs = requests(37, 10)
    server = serving.FrontendServer(torch, budget_bytes=1 << 30, max_clips=32, tables=2)
    ref = run(server, reqs)
    pageable = []
    for r in reqs:
        q = serving.Request(rid=r.rid + 1000, clips=[c.clone() for c in r.clips], rates=list(r.rates), arrival=0.0)
        assert not q.clips[0].is_pinned()
        pageable.append(q)
    for q in pageable:
        serving.attach_outputs(torch, server, q)
        q.outputs = [o.clone() for o in q.outputs]   # pageable outputs too
        q._args = None
    done = server.run(pageable)
    torch.cuda.synchronize()
    got = {q.rid - 1000: q.outputs for q in done}
    for r in reqs:
        for a, b in zip(ref[r.rid], got[r.rid]):
            assert torch.equal(a, b)
    server.close()
