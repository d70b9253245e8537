"""Continuous-batching server for the multi-rate audio front end (resample -> pre-emphasis -> STFT ->
mel -> decibels per clip).

Requests (1..k mono clips at any input rate) arrive at arbitrary times.  The server

* admits a request when the clips' device buffers (input at its rate, the 16 kHz signal, the
  decibel output) fit in a fixed device-memory budget, carved from one arena allocated once;
* uploads the request's clips from pinned host memory on a copy stream;
* runs steps on a compute stream: each step takes every uploaded, not yet processed clip (up to
  `max_clips`), writes their buffer addresses into a device clip table and replays a CUDA graph of
  one `rppb_frontend_clips_gpu` call (the table is read on the device, so one captured graph serves
  every batch composition); up to `tables` steps are in flight, and requests that arrive while a
  step runs join the next one;
* copies each finished request's outputs back on the copy stream and frees its buffers.

Every clip's result depends only on that clip (the kernels index clips through the table), so a
request gives the same bits alone and in any mix — tests/test_gpu_serving.py checks it.
Timing of requests uses the host clock (time.perf_counter) from arrival to the completion of the
output copy.
"""
import ctypes
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import lib
from .types import RppbFrontendParams, frontend_params

ALIGN = 256


class RppbClip(ctypes.Structure):
    _fields_ = [("src", ctypes.c_void_p), ("work", ctypes.c_void_p), ("dst", ctypes.c_void_p),
                ("length", ctypes.c_int32), ("inRate", ctypes.c_float), ("dstStride", ctypes.c_int32),
                ("pad", ctypes.c_int32)]


assert ctypes.sizeof(RppbClip) == 40


class Arena:
    """First-fit allocator over [0, size) in ALIGN-byte units (offsets into one device buffer)."""

    def __init__(self, size):
        self.size = size
        self.free = [(0, size)]          # sorted (offset, length)
        self.used = 0

    def alloc(self, nbytes):
        nbytes = (nbytes + ALIGN - 1) // ALIGN * ALIGN
        for i, (o, l) in enumerate(self.free):
            if l >= nbytes:
                if l == nbytes:
                    self.free.pop(i)
                else:
                    self.free[i] = (o + nbytes, l - nbytes)
                self.used += nbytes
                return o, nbytes
        return None

    def release(self, off, nbytes):
        self.used -= nbytes
        self.free.append((off, nbytes))
        self.free.sort()
        merged = []
        for o, l in self.free:
            if merged and merged[-1][0] + merged[-1][1] == o:
                merged[-1] = (merged[-1][0], merged[-1][1] + l)
            else:
                merged.append((o, l))
        self.free = merged


@dataclass
class Request:
    rid: int
    clips: list                   # pinned torch float32 tensors (mono)
    rates: list
    arrival: float                # host clock
    outputs: list = field(default_factory=list)   # pinned host tensors [numFilter][frames]
    frames: list = field(default_factory=list)
    blocks: list = field(default_factory=list)    # arena (offset, bytes) per clip
    done_clips: int = 0
    upload_event: object = None
    finish: float = None


class FrontendServer:
    def __init__(self, torch, budget_bytes=40 << 30, max_clips=256, tables=4, out_rate=16000.0, lut=None,
                 params=None, preemph=0.97, capture=True):
        from .windows import kaiser_sinc
        self.torch = torch
        self.dev = torch.device("cuda")
        self.L = lib.load()
        self.params = params or frontend_params()
        self.out_rate = float(out_rate)
        self.preemph = float(preemph)
        lut, self.scale, self.center, self.lobes = lut or kaiser_sinc(16)
        self.lut = torch.from_numpy(np.ascontiguousarray(lut)).to(self.dev)
        self.arena_buf = torch.empty(budget_bytes, dtype=torch.uint8, device=self.dev)
        self.base = self.arena_buf.data_ptr()
        self.arena = Arena(budget_bytes)
        self.max_clips = max_clips
        self.compute = torch.cuda.Stream()
        self.copy = torch.cuda.Stream()
        self.handle = lib.Handle(batch_size=max_clips, stream=self.compute.cuda_stream)
        self.ntables = tables
        self.host_tables = [torch.zeros(max_clips * ctypes.sizeof(RppbClip), dtype=torch.uint8).pin_memory()
                            for _ in range(tables)]
        self.dev_tables = [torch.zeros(max_clips * ctypes.sizeof(RppbClip), dtype=torch.uint8, device=self.dev)
                           for _ in range(tables)]
        self.graphs = [None] * tables
        self.capture = capture
        self.table_busy = [None] * tables         # event of the step using table i
        self.pending = deque()                    # submitted, not admitted
        self.ready = deque()                      # (request, clip index) uploaded, waiting for a step
        self.inflight = deque()                   # (event, table, [(request, clip)])
        self.completed = []
        self.next_table = 0

    # ---------------------------------------------------------------- buffers
    def _frames(self, length, rate):
        p = self.params
        lr = length if rate == self.out_rate else int(np.ceil(np.float32(np.float32(length) * np.float32(self.out_rate))
                                                              / np.float32(rate)))
        if p.centerWindows:
            return lr, lr // p.windowStep + 1
        return lr, max(0, (lr - p.windowLength) // p.windowStep + 1)

    def _clip_bytes(self, length, rate):
        lr, f = self._frames(length, rate)
        nf = self.params.numFilter
        return [length * 4, lr * 4 + 16, nf * max(f, 1) * 4], f

    def submit(self, request):
        request.done_clips = 0
        request.finish = None
        request.blocks = []
        request.upload_event = None
        self.pending.append(request)

    def _admit(self):
        torch = self.torch
        while self.pending:
            r = self.pending[0]
            need = []
            for c, rate in zip(r.clips, r.rates):
                sizes, f = self._clip_bytes(c.numel(), rate)
                need.append((sizes, f))
            blocks = []
            ok = True
            for sizes, _ in need:
                got = self.arena.alloc(sum((s + ALIGN - 1) // ALIGN * ALIGN for s in sizes))
                if got is None:
                    ok = False
                    break
                blocks.append(got)
            if not ok:
                for b in blocks:
                    self.arena.release(*b)
                return   # FIFO admission: wait for memory to free up
            self.pending.popleft()
            r.blocks = blocks
            r.frames = [f for _, f in need]
            with torch.cuda.stream(self.copy):
                for c, (off, _) in zip(r.clips, blocks):
                    dst = self.arena_buf[off:off + c.numel() * 4].view(torch.float32)
                    dst.copy_(c, non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(self.copy)
            r.upload_event = ev
            for i in range(len(r.clips)):
                self.ready.append((r, i))

    # ---------------------------------------------------------------- steps
    def _launch(self, table_idx, n):
        """Clip table i -> one rppb_frontend_clips_gpu over max_clips entries (unused entries length 0)."""
        L = self.L
        st = L.rppb_frontend_clips_gpu(self.dev_tables[table_idx].data_ptr(), self.max_clips, self.out_rate,
                                       self.lut.data_ptr(), int(self.lut.numel()), self.scale, self.center,
                                       int(self.lobes), self.preemph, ctypes.byref(self.params), self.handle.value)
        if st != 0:
            raise RuntimeError(f"rppb_frontend_clips_gpu failed: {st} {lib.last_error()}")

    def _run_table(self, table_idx):
        torch = self.torch
        with torch.cuda.stream(self.compute):
            self.dev_tables[table_idx].copy_(self.host_tables[table_idx], non_blocking=True)
            if not self.capture:
                self._launch(table_idx, self.max_clips)
                return
            g = self.graphs[table_idx]
            if g is None:
                # one uncaptured call sizes the handle workspace, then capture copy + call
                self._launch(table_idx, self.max_clips)
                self.compute.synchronize()
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=self.compute):
                    self.dev_tables[table_idx].copy_(self.host_tables[table_idx], non_blocking=True)
                    self._launch(table_idx, self.max_clips)
                self.graphs[table_idx] = g
            g.replay()

    def _step(self):
        if not self.ready:
            return False
        t = self.next_table
        if self.table_busy[t] is not None and not self.table_busy[t].query():
            return False
        torch = self.torch
        batch = []
        waits = set()
        while self.ready and len(batch) < self.max_clips:
            r, i = self.ready[0]
            if not r.upload_event.query():
                break
            self.ready.popleft()
            batch.append((r, i))
            waits.add(id(r.upload_event))
        if not batch:
            return False
        table = (RppbClip * self.max_clips).from_address(self.host_tables[t].data_ptr())
        ctypes.memset(ctypes.addressof(table), 0, ctypes.sizeof(table))
        nf = self.params.numFilter
        for k, (r, i) in enumerate(batch):
            off, _ = r.blocks[i]
            c = r.clips[i]
            sizes, f = self._clip_bytes(c.numel(), r.rates[i])
            a0 = self.base + off
            a1 = a0 + (sizes[0] + ALIGN - 1) // ALIGN * ALIGN
            a2 = a1 + (sizes[1] + ALIGN - 1) // ALIGN * ALIGN
            e = table[k]
            e.src, e.work, e.dst = a0, a1, a2
            e.length, e.inRate, e.dstStride = c.numel(), float(r.rates[i]), max(f, 1)
        self._run_table(t)
        ev = torch.cuda.Event()
        ev.record(self.compute)
        self.table_busy[t] = ev
        self.inflight.append((ev, batch))
        self.next_table = (t + 1) % self.ntables
        return True

    def _retire(self):
        torch = self.torch
        while self.inflight and self.inflight[0][0].query():
            ev, batch = self.inflight.popleft()
            nf = self.params.numFilter
            for r, i in batch:
                off, _ = r.blocks[i]
                c = r.clips[i]
                sizes, f = self._clip_bytes(c.numel(), r.rates[i])
                a2 = off + (sizes[0] + ALIGN - 1) // ALIGN * ALIGN + (sizes[1] + ALIGN - 1) // ALIGN * ALIGN
                out = self.arena_buf[a2:a2 + nf * max(f, 1) * 4].view(torch.float32).view(nf, max(f, 1))
                with torch.cuda.stream(self.copy):
                    self.copy.wait_event(ev)
                    r.outputs[i].copy_(out, non_blocking=True)
                r.done_clips += 1
                if r.done_clips == len(r.clips):
                    with torch.cuda.stream(self.copy):
                        fin = torch.cuda.Event()
                        fin.record(self.copy)
                    self.completed.append((r, fin))

    def _finish(self):
        keep = []
        now = None
        for r, fin in self.completed:
            if fin.query():
                now = now or time.perf_counter()
                r.finish = now
                for b in r.blocks:
                    self.arena.release(*b)
                r.blocks = []
                self.done.append(r)
            else:
                keep.append((r, fin))
        self.completed = keep

    def poll(self):
        """One scheduling round: finish, retire, admit, step."""
        self._finish()
        self._retire()
        self._admit()
        while self._step():
            pass

    def idle(self):
        return not (self.pending or self.ready or self.inflight or self.completed)

    def run(self, requests, arrivals=None):
        """Serves `requests` (submitted at host times `arrivals`, seconds from start; None = all at
        once) and returns them completed, with `.arrival` and `.finish` set."""
        self.done = []
        t0 = time.perf_counter()
        order = list(range(len(requests)))
        k = 0
        while k < len(order) or not self.idle():
            now = time.perf_counter() - t0
            while k < len(order) and (arrivals is None or arrivals[k] <= now):
                r = requests[order[k]]
                r.arrival = t0 + (arrivals[k] if arrivals is not None else 0.0)
                self.submit(r)
                k += 1
            self.poll()
        return self.done


def make_request(torch, rid, rng, max_clips=8, rates=(16000.0, 44100.0, 48000.0), median_s=2.0, sigma=0.6,
                 max_s=30.0, num_filter=128):
    """configs[4] request: 1..max_clips mono clips, durations log-normal (median 2 s, sigma 0.6,
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
    req = Request(rid=rid, clips=clips, rates=rs, arrival=0.0)
    return req


def attach_outputs(torch, server, req):
    """Pinned host outputs [numFilter][frames] for each clip of `req`."""
    nf = server.params.numFilter
    req.outputs = []
    for c, rate in zip(req.clips, req.rates):
        _, f = server._frames(c.numel(), rate)
        req.outputs.append(torch.empty((nf, max(f, 1)), dtype=torch.float32).pin_memory())
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
        clips, rates = [], []
        for _ in range(k):
            rate = self.rates[int(rng.integers(0, len(self.rates)))]
            lst = self.clips[rate]
            clips.append(lst[int(rng.integers(0, len(lst)))])
            rates.append(rate)
        return Request(rid=rid, clips=clips, rates=rates, arrival=0.0)


def clip_seconds(req):
    return sum(c.numel() / r for c, r in zip(req.clips, req.rates))


def measure(torch, server, pool, rng, n_requests, rate_per_s=None):
    """Serves n_requests (all at t=0 when rate_per_s is None, else Poisson arrivals at rate_per_s)
    and returns (clip-s/s over the run, latencies in ms)."""
    reqs = [attach_outputs(torch, server, pool.request(i, rng)) for i in range(n_requests)]
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
