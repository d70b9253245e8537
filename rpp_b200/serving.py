"""Continuous-batching server for the multi-rate audio front end (resample -> pre-emphasis -> STFT ->
mel -> decibels per clip): the Python face of the native server in include/rppb_server.h
(rpp_b200/csrc/server.cu).

Requests (1..k mono clips at any input rate, pinned host tensors) arrive at arbitrary times.  The
native scheduler thread admits them first come, first served into a fixed device arena (the memory
budget), copies their clips in on an upload stream (one copy kernel per admission round over the
pinned clips), runs steps that replay one captured graph of the front end over a clip table (every
uploaded clip not yet processed joins the next step; several steps in flight), copies each finished
clip's decibels out on a download stream (one copy kernel per round) and reports the request
complete.  A step runs the fused front end (rppb_frontend_clips_gpu) or, for comparison, the plain
FP32 path (resample, then the four rppt_*_gpu calls on a batch buffer).

Every clip's result depends only on that clip (the kernels index clips through the table), so a
request gives the same bits alone and in any mix -- tests/test_gpu_serving.py checks it.  Latency is
measured on the steady clock from a request's arrival to the end of its last output copy.
"""
import ctypes
import time
from dataclasses import dataclass, field

import numpy as np

from . import lib
from .types import RppbCompletion, RppbServerConfig, frontend_params


@dataclass
class Request:
    rid: int
    clips: list                   # pinned torch float32 tensors (mono)
    rates: list
    arrival: float                # host clock (time.perf_counter), set when submitted
    outputs: list = field(default_factory=list)   # pinned host tensors [numFilter][frames]
    finish: float = None
    _args: tuple = None           # ctypes arrays handed to rppb_server_submit


class FrontendServer:
    """Owns one native server (rppb_server_create) on the current device."""

    def __init__(self, torch, budget_bytes=40 << 30, max_clips=256, tables=4, out_rate=16000.0, lut=None,
                 params=None, preemph=0.97, plain=False, max_samples=0):
        """plain=True runs each step through the plain FP32 path (resample, then the four rppt_*_gpu
        calls on a batch buffer of max_clips rows of max_samples samples at out_rate; 0 = 30 s) instead
        of the fused front end."""
        from .windows import kaiser_sinc
        self.torch = torch
        self.L = lib.load()
        self.params = params or frontend_params()
        self.out_rate = float(out_rate)
        lut, scale, center, lobes = lut or kaiser_sinc(16)
        self._lut = np.ascontiguousarray(lut, np.float32)
        cfg = RppbServerConfig()
        cfg.budgetBytes = int(budget_bytes)
        cfg.maxClipsPerStep = int(max_clips)
        cfg.tables = int(tables)
        cfg.outRate = self.out_rate
        cfg.lookup = self._lut.ctypes.data
        cfg.lookupSize = int(self._lut.size)
        cfg.scale, cfg.center, cfg.lobes = float(scale), float(center), int(lobes)
        cfg.preemphCoeff = float(preemph)
        cfg.params = self.params
        cfg.plainChain = 1 if plain else 0
        cfg.maxSamples = int(max_samples)
        self.plain = bool(plain)
        self._cfg = cfg
        self._h = ctypes.c_void_p()
        st = self.L.rppb_server_create(ctypes.byref(self._h), ctypes.byref(cfg))
        if st != 0:
            raise RuntimeError(f"rppb_server_create failed: {st} {lib.last_error()}")
        self._byid = {}
        self._buf = (RppbCompletion * 256)()

    def close(self):
        if self._h:
            self.L.rppb_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def frames(self, length, rate):
        return int(self.L.rppb_server_frames(self._h, int(length), float(rate)))

    def _frames(self, length, rate):
        """(outRate length in the reference's float arithmetic, frames)."""
        lr = length if rate == self.out_rate else int(np.ceil(np.float32(np.float32(length) * np.float32(self.out_rate))
                                                              / np.float32(rate)))
        return lr, self.frames(length, rate)

    def arena_used(self):
        return int(self.L.rppb_server_arena_used(self._h))

    def prepare(self, request):
        """Builds the pointer arrays of a request once (keeps submission cheap)."""
        k = len(request.clips)
        P = ctypes.c_void_p * k
        request._args = (P(*[c.data_ptr() for c in request.clips]),
                         (ctypes.c_int32 * k)(*[c.numel() for c in request.clips]),
                         (ctypes.c_float * k)(*[float(r) for r in request.rates]),
                         P(*[o.data_ptr() for o in request.outputs]), k)
        return request

    def submit(self, request):
        if request._args is None:
            self.prepare(request)
        rid = ctypes.c_uint64()
        a = request._args
        st = self.L.rppb_server_submit(self._h, a[0], a[1], a[2], a[3], a[4], ctypes.byref(rid))
        if st != 0:
            raise RuntimeError(f"rppb_server_submit failed: {st} {lib.last_error()}")
        request.finish = None
        self._byid[rid.value] = request
        return rid.value

    def poll(self):
        """Completed requests since the last poll, with .finish set (perf_counter seconds)."""
        out = []
        while True:
            n = ctypes.c_int32()
            st = self.L.rppb_server_poll(self._h, self._buf, len(self._buf), ctypes.byref(n))
            if st != 0:
                raise RuntimeError(f"rppb_server_poll failed: {st} {lib.last_error()}")
            for i in range(n.value):
                c = self._buf[i]
                r = self._byid.pop(c.id)
                r.finish = c.finishNs * 1e-9
                out.append(r)
            if n.value < len(self._buf):
                return out

    def run(self, requests, arrivals=None):
        """Serves `requests` (arriving at host times `arrivals`, seconds from start; None = all at
        once) and returns them completed, with `.arrival` and `.finish` on the steady clock."""
        for r in requests:
            if r._args is None:
                self.prepare(r)
        done = []
        t0 = time.perf_counter()
        k = 0
        while k < len(requests) or len(done) < len(requests):
            now = time.perf_counter() - t0
            while k < len(requests) and (arrivals is None or arrivals[k] <= now):
                r = requests[k]
                r.arrival = t0 + (arrivals[k] if arrivals is not None else 0.0)
                self.submit(r)
                k += 1
            done.extend(self.poll())
            if k < len(requests) and arrivals is not None:
                wait = arrivals[k] - (time.perf_counter() - t0)
                if wait > 2e-4:
                    time.sleep(wait - 1e-4)
        return done


def make_request(torch, rid, rng, max_clips=8, rates=(16000.0, 44100.0, 48000.0), median_s=2.0, sigma=0.6,
                 max_s=30.0, num_filter=128):
    """One serving request: 1..max_clips mono clips, durations log-normal (median 2 s, sigma 0.6,
    clipped to 0.1..max_s s), rates uniform over `rates`, same signal model as the other configs."""
    from . import synth
    k = int(rng.integers(1, max_clips + 1))
    clips, rs, outs = [], [], []
    for _ in range(k):
        rate = float(rng.choice(rates))
        dur = float(np.clip(rng.lognormal(np.log(median_s), sigma), 0.1, max_s))
        n = max(1, int(dur * rate))
        x, _ = synth.mono_batch(1, [n], rng, rate=int(rate))
        clips.append(torch.from_numpy(x[0]).pin_memory())
        rs.append(rate)
    return Request(rid=rid, clips=clips, rates=rs, arrival=0.0)


def attach_outputs(torch, server, req):
    """Pinned host outputs [numFilter][frames] for each clip of `req`."""
    nf = server.params.numFilter
    req.outputs = [torch.empty((nf, max(server.frames(c.numel(), rate), 1)), dtype=torch.float32).pin_memory()
                   for c, rate in zip(req.clips, req.rates)]
    req._args = None
    return req


class ClipPool:
    """Pre-generated pinned clips for request streams: `per_rate` clips per input rate with
    log-normal durations (median 2 s, sigma 0.6, clipped to 0.1..max_s s); requests draw from it so
    generating audio stays out of the serving loop."""

    def __init__(self, torch, rng, rates=(16000.0, 44100.0, 48000.0), per_rate=48, median_s=2.0, sigma=0.6,
                 max_s=30.0):
        from . import synth
        self.rates = list(rates)
        self.clips = {}
        for rate in self.rates:
            lst = []
            for _ in range(per_rate):
                dur = float(np.clip(rng.lognormal(np.log(median_s), sigma), 0.1, max_s))
                n = max(1, int(dur * rate))
                x, _ = synth.mono_batch(1, [n], rng, rate=int(rate))
                lst.append(torch.from_numpy(x[0]).pin_memory())
            self.clips[rate] = lst

    def request(self, rid, rng, max_clips=8):
        k = int(rng.integers(1, max_clips + 1))
        clips, rates, keys = [], [], []
        for _ in range(k):
            rate = self.rates[int(rng.integers(0, len(self.rates)))]
            lst = self.clips[rate]
            i = int(rng.integers(0, len(lst)))
            clips.append(lst[i])
            rates.append(rate)
            keys.append((rate, i))
        r = Request(rid=rid, clips=clips, rates=rates, arrival=0.0)
        r.keys = keys
        return r

    def attach_shared_outputs(self, torch, server, req):
        """Outputs of `req` from one pinned buffer per pool clip, allocated on first use: requests that
        share a clip write the same values to the same buffer, so long request streams need no new
        host memory per request."""
        cache = self.__dict__.setdefault("_outs", {})
        nf = server.params.numFilter
        outs = []
        for key, c, rate in zip(req.keys, req.clips, req.rates):
            if key not in cache:
                cache[key] = torch.empty((nf, max(server.frames(c.numel(), rate), 1)),
                                         dtype=torch.float32).pin_memory()
            outs.append(cache[key])
        req.outputs = outs
        req._args = None
        return req


def clip_seconds(req):
    return sum(c.numel() / r for c, r in zip(req.clips, req.rates))


def measure(torch, server, pool, rng, n_requests, rate_per_s=None):
    """Serves n_requests (all at t=0 when rate_per_s is None, else Poisson arrivals at rate_per_s)
    and returns (clip-s/s over the run, latencies in ms)."""
    reqs = [pool.attach_shared_outputs(torch, server, pool.request(i, rng)) for i in range(n_requests)]
    if rate_per_s is None:
        arrivals = None
    else:
        arrivals = list(np.cumsum(rng.exponential(1.0 / rate_per_s, n_requests)))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    done = server.run(reqs, arrivals)
    t1 = time.perf_counter()
    lat = np.array([(r.finish - r.arrival) * 1e3 for r in done])
    total = sum(clip_seconds(r) for r in done)
    span = (t1 - t0) if arrivals is None else max(t1 - t0, 1e-9)
    return total / span, lat
