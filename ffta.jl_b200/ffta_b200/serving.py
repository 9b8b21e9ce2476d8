"""Continuous-batching transform server over the sm_100a library.

FFTA.jl has no serving layer; this module is a request loop on top of the
drop-in path.  Requests are (length n, element type,
direction, batch count, seed, arrival time).  The loop:

* admits waiting requests in arrival order while their device bytes (input +
  output + multi-pass scratch) fit a budget (100 GB by default), and releases
  a request's bytes when it completes;
* keeps plans (twiddle/chirp tables, scratch) resident, keyed by
  (n, type, direction) -- and the batch for multi-pass lengths;
* packs every admitted small single-pass request -- any mix of lengths,
  types and directions -- into one work-descriptor launch per kernel variant
  (each block looks up its request's descriptor); multi-pass lengths and
  large requests (2^18 elements or more) run their cached plans, each plan on
  a stream of its own so different plans overlap;
* rotates launches over several CUDA streams and dispatches whatever arrived
  while earlier launches run, as soon as a stream is free (continuous
  batching); completions are timed with CUDA events on the device clock.

The loop itself is native (fb_server_* in the C ABI); `Server` here drives it
with arrivals and polls.

`run_one_by_one` is the plain path it is compared with: each request, on
arrival, runs its own plan and is synchronised before the next one starts.

Both paths read the same device-resident inputs (generated from the
per-request seeds before timing) so that what is compared is the serving of
transforms, not data generation.
"""
from __future__ import annotations

import bisect
import collections
import ctypes
import dataclasses
import math
import time

import numpy as np

from . import (_lib, _check, plan_fft, plan_bfft, FB_SERVER_NO_GRAPHS, FB_SERVER_NO_PERSISTENT,
               FB_SERVER_SERIAL)

ELEM = {"c64": 8, "c128": 16}


@dataclasses.dataclass
class Request:
    rid: int
    n: int
    kind: str  # "c64" (ComplexF32) or "c128" (ComplexF64)
    dir: int  # -1 forward, +1 backward
    batch: int
    seed: int
    arrival: float  # seconds from the start of the run
    done: float = math.nan  # completion time, seconds from the start

    @property
    def bytes_io(self) -> int:
        return 2 * self.n * self.batch * ELEM[self.kind]

    @property
    def flops(self) -> float:
        return 5.0 * self.n * math.log2(max(self.n, 2)) * self.batch


# ----------------------------------------------------------------- traces
def _is_prime(v: int) -> bool:
    if v < 2:
        return False
    if v % 2 == 0:
        return v == 2
    f = 3
    while f * f <= v:
        if v % f == 0:
            return False
        f += 2
    return True


def _smooth_near(target: float, primes, need=None) -> int:
    """The product of `primes` closest to target (log scale), using `need`."""
    best, bestd = 1, float("inf")
    lt = math.log(target)

    def rec(i, v):
        nonlocal best, bestd
        if v > target * 2:
            return
        if i == len(primes):
            if need is not None and v % need:
                return
            d = abs(math.log(v) - lt)
            if d < bestd:
                best, bestd = v, d
            return
        p = primes[i]
        while v <= target * 2:
            rec(i + 1, v)
            v *= p

    rec(0, 1)
    return best


def make_trace(count: int, rate: float, seed: int = 0, n_min: int = 64, n_max: int = 2 ** 20,
               batch_max: int = 512, mix=(0.5, 0.2, 0.15, 0.15), c64_frac=0.2):
    """Requests of the serving configuration.

    Length log-uniform on [n_min, n_max] and rounded into its class: 50 % powers
    of two, 20 % 2^a 3^b (b >= 1), 15 % other smooth composites (a factor 5 or
    7), 15 % primes; direction forward/backward 50/50; ComplexF32 80 % /
    ComplexF64 20 %; batch uniform on 1..batch_max; Poisson arrivals at `rate`
    requests per second; one seed per request.
    """
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    lo, hi = math.log(n_min), math.log(n_max)
    for i in range(count):
        t += rng.exponential(1.0 / rate) if rate > 0 else 0.0
        target = math.exp(rng.uniform(lo, hi))
        c = rng.choice(4, p=list(mix))
        if c == 0:
            n = 2 ** int(round(math.log2(target)))
        elif c == 1:
            n = _smooth_near(target, [2, 3], need=3)
        elif c == 2:
            n = _smooth_near(target, [2, 3, 5, 7], need=int(rng.choice([5, 7])))
        else:
            n = int(target)
            while not _is_prime(n):
                n += 1
        n = int(min(max(n, n_min if c != 3 else 2), n_max * 2))
        kind = "c128" if rng.random() < c64_frac else "c64"
        out.append(Request(i, n, kind, -1 if rng.random() < 0.5 else 1,
                           int(rng.integers(1, batch_max + 1)), int(rng.integers(0, 2 ** 31)), t))
    return out


def make_inputs(trace, device):
    """Device-resident complex-normal inputs, one per request, from its seed."""
    import torch
    xs = []
    for r in trace:
        g = torch.Generator(device=device)
        g.manual_seed(r.seed)
        rdt = torch.float32 if r.kind == "c64" else torch.float64
        shape = (r.batch, r.n)
        xs.append(torch.complex(torch.randn(shape, generator=g, device=device, dtype=rdt),
                                torch.randn(shape, generator=g, device=device, dtype=rdt)))
    return xs


# ------------------------------------------------------------------ plans
class PlanCache:
    """Resident plans: grouped (n, kind, dir) and per-batch (n, kind, dir, batch)."""

    def __init__(self):
        self.group = {}
        self.single = {}

    def _make(self, n, kind, direction, batch):
        import torch
        dt = torch.complex64 if kind == "c64" else torch.complex128
        x = torch.empty((batch, n), dtype=dt, device="cuda")
        p = (plan_fft if direction < 0 else plan_bfft)(x.T, 1)
        p._cplan(x.T, x.T)  # build the device schedule now
        return p, p._cplans[next(iter(p._cplans))]

    def grouped(self, n, kind, direction):
        key = (n, kind, direction)
        if key not in self.group:
            p, h = self._make(n, kind, direction, 1)
            buf = ctypes.create_string_buffer(4096)
            _check(_lib.lib.fb_plan_describe(h, buf, len(buf)))
            ok = "FAST(" in buf.value.decode() and buf.value.decode().count("(") == 1
            self.group[key] = (p, h, ok)
        return self.group[key]

    def single_plan(self, n, kind, direction, batch):
        key = (n, kind, direction, batch)
        if key not in self.single:
            self.single[key] = self._make(n, kind, direction, batch)
        return self.single[key]

    def scratch_bytes(self, r: Request) -> int:
        p, h = self.single_plan(r.n, r.kind, r.dir, r.batch) if not self.grouped(
            r.n, r.kind, r.dir)[2] else self.grouped(r.n, r.kind, r.dir)[:2]
        v = ctypes.c_size_t()
        _check(_lib.lib.fb_plan_device_bytes(h, ctypes.byref(v)))
        return int(v.value)


def warm_plans(trace, cache: PlanCache):
    for r in trace:
        _, _, ok = cache.grouped(r.n, r.kind, r.dir)
        if not ok:
            cache.single_plan(r.n, r.kind, r.dir, r.batch)


# ------------------------------------------------------------- execution
def _stream_ptr(s):
    return ctypes.c_void_p(s.cuda_stream)


def _run_single(cache, r, x, y, stream):
    _, h, ok = cache.grouped(r.n, r.kind, r.dir)
    if ok:
        ins = (ctypes.c_void_p * 1)(x.data_ptr())
        outs = (ctypes.c_void_p * 1)(y.data_ptr())
        bs = (ctypes.c_int64 * 1)(r.batch)
        _check(_lib.lib.fb_execute_grouped(h, 1, ins, outs, bs, _stream_ptr(stream)))
    else:
        _, hs = cache.single_plan(r.n, r.kind, r.dir, r.batch)
        _check(_lib.lib.fb_execute(hs, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                                   _stream_ptr(stream)))


def _stats(trace, wall, label):
    lat = np.array([r.done - r.arrival for r in trace])
    fl = sum(r.flops for r in trace)
    by = sum(r.bytes_io for r in trace)
    span = max(r.done for r in trace) - min(r.arrival for r in trace)
    return {
        "path": label, "requests": len(trace), "wall_s": wall, "span_s": span,
        "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
        "mean_ms": float(lat.mean() * 1e3),
        "throughput_req_s": len(trace) / span, "GFLOP/s": fl / span / 1e9, "GB/s": by / span / 1e9,
    }


def run_one_by_one(trace, xs, ys, cache: PlanCache):
    """One launch per request, each synchronised before the next (the plain path)."""
    import torch
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for r, x, y in zip(trace, xs, ys):
        while True:  # wait for the arrival (sleep long gaps, spin short ones)
            gap = r.arrival - (time.perf_counter() - t0)
            if gap <= 0:
                break
            if gap > 2e-4:
                time.sleep(gap - 1e-4)
        _run_single(cache, r, x, y, stream)
        stream.synchronize()
        r.done = time.perf_counter() - t0
    return _stats(trace, time.perf_counter() - t0, "one_launch_per_request")


class Server:
    """Driver of the library's native server (fb_server_*): submits each
    request when it arrives and polls for completions.  Admission, packing
    into work-descriptor launches and stream rotation happen in the library.
    Completion times come from CUDA events on the device clock, counted from
    the server's creation (the run's time origin).  With `graphs`, a
    multi-pass request that recurs on the same buffers is replayed from a
    CUDA graph captured on its second occurrence."""

    KIND = {"c64": _lib.FB_C32, "c128": _lib.FB_C64}
    NSTATS = 13

    def __init__(self, budget_bytes: float = 100e9, nstreams: int = 4, graphs: bool = True,
                 resident: bool = True, serial: bool = False):
        self.budget = budget_bytes
        self.nstreams = nstreams
        self.h = ctypes.c_void_p()
        self.serial = serial
        flags = ((0 if graphs else FB_SERVER_NO_GRAPHS) |
                 (0 if resident else FB_SERVER_NO_PERSISTENT) | (FB_SERVER_SERIAL if serial else 0))
        _check(_lib.lib.fb_server_create(ctypes.byref(self.h), float(budget_bytes), nstreams,
                                         flags))

    def stats(self):
        st = (ctypes.c_int64 * self.NSTATS)()
        _check(_lib.lib.fb_server_stats(self.h, st, self.NSTATS))
        return list(st)

    def __del__(self):
        try:
            _lib.lib.fb_server_destroy(self.h)
        except Exception:
            pass

    def run(self, trace, xs, ys):
        """Serve `trace` (arrival times relative to the call); the server's
        plans stay resident between runs."""
        import torch
        torch.cuda.synchronize()
        h = self.h
        st0 = self.stats()
        n = len(trace)
        # request fields as arrays, so that everything that has arrived is
        # submitted with one call
        a_n = np.array([r.n for r in trace], dtype=np.int64)
        a_t = np.array([self.KIND[r.kind] for r in trace], dtype=np.int32)
        a_d = np.array([r.dir for r in trace], dtype=np.int32)
        a_b = np.array([r.batch for r in trace], dtype=np.int64)
        a_in = (ctypes.c_void_p * n)(*[x.data_ptr() for x in xs[:n]])
        a_out = (ctypes.c_void_p * n)(*[y.data_ptr() for y in ys[:n]])
        tickets = np.zeros(n, dtype=np.int64)
        arrivals = np.array([r.arrival for r in trace])
        cap = 4096
        tk = np.zeros(cap, dtype=np.int64)
        tm = np.zeros(cap, dtype=np.float64)
        cnt = ctypes.c_int64()
        i64 = ctypes.POINTER(ctypes.c_int64)
        i32 = ctypes.POINTER(ctypes.c_int32)
        vpp = ctypes.POINTER(ctypes.c_void_p)
        sz = ctypes.sizeof(ctypes.c_void_p)
        done = np.full(n, np.nan)
        base = None
        _check(_lib.lib.fb_server_reset_clock(h))
        t0 = time.perf_counter()
        nxt, ndone = 0, 0
        try:
            while ndone < n:
                now = time.perf_counter() - t0
                upto = int(np.searchsorted(arrivals, now, side="right"))
                if upto > nxt:
                    k = upto - nxt
                    _check(_lib.lib.fb_server_submit_many(
                        h, k, a_n[nxt:].ctypes.data_as(i64), a_t[nxt:].ctypes.data_as(i32),
                        a_d[nxt:].ctypes.data_as(i32), a_b[nxt:].ctypes.data_as(i64),
                        ctypes.cast(ctypes.addressof(a_in) + nxt * sz, vpp),
                        ctypes.cast(ctypes.addressof(a_out) + nxt * sz, vpp),
                        tickets[nxt:].ctypes.data_as(i64)))
                    if base is None:
                        base = int(tickets[0])  # tickets are consecutive
                    nxt = upto
                _check(_lib.lib.fb_server_poll(h, cap, tk.ctypes.data_as(i64),
                                               tm.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                               ctypes.byref(cnt)))
                c = cnt.value
                if c:
                    done[tk[:c] - base] = tm[:c] * 1e-3
                ndone += c
                if cnt.value == 0 and nxt < n and ndone == nxt:
                    # idle until the next arrival: sleep only for gaps well above
                    # the OS timer's overshoot (tens of microseconds), else spin
                    dt = arrivals[nxt] - (time.perf_counter() - t0)
                    if dt > 2e-4:
                        time.sleep(min(dt - 1e-4, 0.0005))
        finally:
            st1 = self.stats()
        for r, d in zip(trace, done):
            r.done = float(d)
        out = _stats(trace, time.perf_counter() - t0, "continuous_batching")
        out.update({"launches": st1[1] - st0[1], "descriptor_launches": st1[2] - st0[2],
                    "max_queue": st1[3], "max_admitted_GB": st1[4] / 1e9,
                    "resident_plans": st1[5], "graph_launches": st1[6] - st0[6],
                    "graph_captures": st1[7] - st0[7], "streams": self.nstreams,
                    "resident_kernel_requests": st1[9] - st0[9],
                    "failed_requests": st1[10] - st0[10]})
        return out


def check_mix_equals_alone(trace, xs, ys_mix, cache: PlanCache):
    """Each request's result in the mix equals its result run alone (bitwise)."""
    import torch
    worst = 0.0
    for r, x, y in zip(trace, xs, ys_mix):
        alone = torch.empty_like(x)
        _run_single(cache, r, x, alone, torch.cuda.current_stream())
        torch.cuda.synchronize()
        d = (alone - y).abs().max().item()
        worst = max(worst, d)
    return worst


# ------------------------------------------------------------ benchmark
def compare_graphs(count=600, seed=13, nstreams=4, repeats=5):
    """Recurring small multi-pass requests (four-step and three-pass Bluestein
    lengths, batch 1..4, below the packing limit, so each runs its cached
    plan: 2-3 kernels), all queued at once, served again and again on the
    same buffers by a server that replays CUDA graphs and by one that
    launches the plans' kernels each time.  Two warm-up runs each (plans,
    then graphs), then the median of `repeats` runs.  Results of the two must
    be equal bit for bit."""
    import torch
    rng = np.random.default_rng(seed)
    lengths = [20000, 32768, 40000, 65536, 65537, 100003, 24576, 50000]
    reqs = [Request(i, int(rng.choice(lengths)), "c128" if rng.random() < 0.2 else "c64",
                    -1 if rng.random() < 0.5 else 1, int(rng.integers(1, 5)),
                    int(rng.integers(0, 2 ** 31)), 0.0) for i in range(count)]
    xs = make_inputs(reqs, "cuda")
    out = {}
    ys_of = {}
    for label, graphs in (("graphs", True), ("no_graphs", False)):
        ys = [torch.empty_like(x) for x in xs]
        srv = Server(100e9, nstreams, graphs=graphs)
        for _ in range(2):
            srv.run([dataclasses.replace(r) for r in reqs], xs, ys)
        runs = [srv.run([dataclasses.replace(r) for r in reqs], xs, ys) for _ in range(repeats)]
        runs.sort(key=lambda st: st["throughput_req_s"])
        out[label] = runs[len(runs) // 2]
        ys_of[label] = ys
        del srv
    diff = max((a - b).abs().max().item() for a, b in zip(ys_of["graphs"], ys_of["no_graphs"]))
    out["throughput_ratio"] = (out["graphs"]["throughput_req_s"] /
                               out["no_graphs"]["throughput_req_s"])
    out["graphs_vs_launches_max_abs_diff"] = diff
    out["notes"] = {"requests": count, "lengths": lengths, "batch": "1..4", "repeats": repeats}
    return out


def compare(count=400, rates=(2000.0,), seed=11, n_max=2 ** 20, batch_max=512,
            max_elems=1 << 22, budget_bytes=100e9, nstreams=4, resident=True):
    """Serve one trace with both paths at each arrival rate of a sweep.

    Requests whose n * batch exceeds `max_elems` get their batch reduced so the
    whole trace's inputs fit on the device next to the outputs (the bounded
    sample of the configuration; the distribution of n is unchanged).  Returns
    {"sweep": [{rate, batched, one_launch_per_request}...], "notes": ...}.
    """
    import torch
    base = make_trace(count, 1.0, seed, n_max=n_max, batch_max=batch_max)
    capped = 0
    for r in base:
        if r.n * r.batch > max_elems:
            r.batch = max(1, max_elems // r.n)
            capped += 1
    cache = PlanCache()
    warm_plans(base, cache)
    xs = make_inputs(base, "cuda")
    ys = [torch.empty_like(x) for x in xs]
    srv = Server(budget_bytes, nstreams, resident=resident)
    # two warm-up passes: resident plans, then graphs of the multi-pass
    # requests (each runs again on the same buffers in every sweep point)
    for _ in range(2):
        srv.run([dataclasses.replace(r, arrival=0.0) for r in base], xs, ys)
    run_one_by_one([dataclasses.replace(r, arrival=0.0) for r in base[:8]], xs[:8], ys[:8], cache)
    worst = check_mix_equals_alone(base[:50], xs[:50], ys[:50], cache)
    sweep = []
    for rate in rates:
        # the same requests, arrivals rescaled to `rate` (rate 0: all at once)
        tr = [dataclasses.replace(r, arrival=(r.arrival / rate if rate > 0 else 0.0))
              for r in base]
        b = srv.run([dataclasses.replace(r) for r in tr], xs, ys)
        p = run_one_by_one([dataclasses.replace(r) for r in tr], xs, ys, cache)
        sweep.append({"rate_req_s": rate if rate > 0 else "all_at_t0", "batched": b,
                      "one_launch_per_request": p,
                      "throughput_ratio": b["throughput_req_s"] / p["throughput_req_s"]})
    notes = {"requests": count, "requests_with_batch_capped": capped,
             "max_elems_per_request": max_elems, "mix_vs_alone_max_abs_diff": worst,
             "distinct_plans": len(cache.group) + len(cache.single)}
    return {"sweep": sweep, "notes": notes}


# ----------------------------------------------------- configuration 5, full
class _Ring:
    """Output space for requests in flight: a ring over one device buffer.
    A request gets the next free span (wrapping to the start); spans are
    released when their request completes."""

    def __init__(self, nbytes: int, device="cuda"):
        import torch
        self.buf = torch.empty(nbytes, dtype=torch.uint8, device=device)
        self.size = nbytes
        self.head = 0
        self.live = {}  # rid -> start
        self.starts = []  # starts of the live spans, ascending
        self.end = {}  # start -> end

    def alloc(self, nbytes: int, rid: int):
        nbytes = (nbytes + 255) // 256 * 256
        if nbytes > self.size:
            raise ValueError("request larger than the output ring")
        for start in (self.head, 0):
            if start + nbytes > self.size:
                continue
            i = bisect.bisect_left(self.starts, start)
            if i < len(self.starts) and self.starts[i] < start + nbytes:
                continue  # a live span starts inside
            if i > 0 and self.end[self.starts[i - 1]] > start:
                continue  # the previous live span reaches into it
            self.starts.insert(i, start)
            self.end[start] = start + nbytes
            self.live[rid] = start
            self.head = start + nbytes
            return start
        return None

    def view(self, start: int, r: "Request"):
        import torch
        dt = torch.complex64 if r.kind == "c64" else torch.complex128
        es = ELEM[r.kind]
        return self.buf[start:start + r.n * r.batch * es].view(dt).view(r.batch, r.n)

    def free(self, rid: int):
        start = self.live.pop(rid, None)
        if start is not None:
            del self.starts[bisect.bisect_left(self.starts, start)]
            del self.end[start]


class _Pools:
    """Device-resident complex-normal input data, one pool per element type,
    each as long as the largest request of its type.  Request r reads
    n*batch consecutive values starting at an offset drawn from its seed
    (inputs drawn from a pool rather than made per request, so that 100k
    requests of up to 2^29 values fit on the device)."""

    def __init__(self, elems, seed: int = 5):
        import torch
        self.elems = dict(elems)  # kind -> values
        self.pool = {}
        for kind, cdt in (("c64", torch.complex64), ("c128", torch.complex128)):
            if self.elems.get(kind, 0) <= 0:
                continue
            g = torch.Generator(device="cuda").manual_seed(seed)
            z = torch.empty(self.elems[kind], dtype=cdt, device="cuda")
            torch.view_as_real(z).normal_(generator=g)  # no temporaries
            self.pool[kind] = z

    def input(self, r: "Request"):
        m = r.n * r.batch
        off = (r.seed % (self.elems[r.kind] - m + 1)) & ~1  # even: 16-byte aligned
        return self.pool[r.kind][off:off + m].view(r.batch, r.n)


def _serve(srv: "Server", trace, pools: _Pools, ring: _Ring, t0_shift=0.0):
    """Drive `srv` with the trace's arrivals; outputs in the ring (a request
    is submitted once it has arrived and its output space is free).  Returns
    per-request completion times (s, device clock) and the run's statistics."""
    import torch
    h = srv.h
    n = len(trace)
    arrivals = np.array([r.arrival for r in trace])
    done = np.full(n, np.nan)
    cap = 4096
    tk = np.zeros(cap, dtype=np.int64)
    tm = np.zeros(cap, dtype=np.float64)
    cnt = ctypes.c_int64()
    ticket_of = {}
    tkt = ctypes.c_int64()
    i64 = ctypes.POINTER(ctypes.c_int64)
    st0 = srv.stats()
    torch.cuda.synchronize()
    _check(_lib.lib.fb_server_reset_clock(h))
    t0 = time.perf_counter()
    nxt, ndone, failed, failed_no_program = 0, 0, 0, 0
    while ndone < n:
        now = time.perf_counter() - t0
        while nxt < n and arrivals[nxt] <= now:
            r = trace[nxt]
            start = ring.alloc(r.n * r.batch * ELEM[r.kind], nxt)
            if start is None:
                break  # output space frees as requests complete
            x = pools.input(r)
            y = ring.view(start, r)
            _check(_lib.lib.fb_server_submit(h, r.n, Server.KIND[r.kind], r.dir, r.batch,
                                             ctypes.c_void_p(x.data_ptr()),
                                             ctypes.c_void_p(y.data_ptr()), ctypes.byref(tkt)))
            ticket_of[tkt.value] = nxt
            nxt += 1
        _check(_lib.lib.fb_server_poll(h, cap, tk.ctypes.data_as(i64),
                                       tm.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                       ctypes.byref(cnt)))
        for j in range(cnt.value):
            k = ticket_of.pop(int(tk[j]))
            done[k] = tm[j] * 1e-3 if tm[j] >= 0 else np.nan
            failed += tm[j] < 0
            failed_no_program += tm[j] == -2.0
            ring.free(k)
        ndone += cnt.value
        if cnt.value == 0 and nxt < n and ndone == nxt:
            dt = arrivals[nxt] - (time.perf_counter() - t0)
            if dt > 2e-4:
                time.sleep(min(dt - 1e-4, 0.0005))
    wall = time.perf_counter() - t0
    st1 = srv.stats()
    for r, d in zip(trace, done):
        r.done = float(d)
    out = _stats([r for r in trace if not math.isnan(r.done)], wall,
                 "serial" if st1[1] and srv.serial else "continuous_batching")
    out.update({"failed": int(failed), "failed_without_program": int(failed_no_program),
                "launches": st1[1] - st0[1],
                "descriptor_launches": st1[2] - st0[2],
                "resident_kernel_requests": st1[9] - st0[9],
                "graph_launches": st1[6] - st0[6], "plans_made": st1[11] - st0[11],
                "plans_released": st1[12] - st0[12], "max_admitted_GB": st1[4] / 1e9})
    return out


def _schedule_class(n: int, kind: str) -> str:
    lmax = 16384 if kind == "c64" else 8192
    if _is_prime(n) and n >= 73:
        return "bluestein"
    return "one_pass" if n <= lmax else "multi_pass"


def compare_config5(count=100000, seed=11, budget_bytes=100e9, nstreams=4,
                    prefix=10000, prefix_rates=(1000.0, 3000.0), sample=240,
                    pool_elems=1 << 29, ring_bytes=48 << 30, reference=None):
    """Configuration 5 at its stated scale: `count` requests (length
    log-uniform 64..2^20 in the class mix, batch 1..512, 80 % ComplexF32,
    forward/backward 50/50), a 100 GB admission budget, served by the
    continuous-batching server and by the same server in serial mode (one
    request at a time, one plan launch each: the one-launch-per-request
    path).  Both start cold (plans made on first use, least recently used
    released), read inputs from a device pool and write into an output ring.

    The full trace runs with every request queued at t0 (saturation); the
    Poisson rate sweep runs on its first `prefix` requests.  Accuracy (when a
    `reference(x, dir)` -- rows of x transformed in FP64 -- is given): a
    stratified sample of `sample` requests (every schedule class and type)
    is served again and its first transform compared with the reference."""
    import torch
    base = make_trace(count, 1.0, seed)
    need = collections.defaultdict(int)
    for r in base:
        need[r.kind] = max(need[r.kind], r.n * r.batch)
    # at least `pool_elems` values, so that small requests read many offsets
    pools = _Pools({k: max(v, min(pool_elems, v * 64)) for k, v in need.items()})
    ring = _Ring(ring_bytes)
    result = {"requests": count, "budget_GB": budget_bytes / 1e9, "sweep": []}
    runs = [("all_at_t0", 0.0, base)] + [(r, r, base[:prefix]) for r in prefix_rates]
    for label, rate, tr in runs:
        point = {"rate_req_s": label, "requests": len(tr)}
        for name, serial in (("batched", False), ("one_launch_per_request", True)):
            srv = Server(budget_bytes, nstreams, serial=serial)
            reqs = [dataclasses.replace(r, arrival=(r.arrival / rate if rate > 0 else 0.0))
                    for r in tr]
            point[name] = _serve(srv, reqs, pools, ring)
            del srv
            torch.cuda.synchronize()
        point["throughput_ratio"] = (point["batched"]["throughput_req_s"] /
                                     point["one_launch_per_request"]["throughput_req_s"])
        result["sweep"].append(point)
    if reference is None:
        return result
    # accuracy on a stratified sample, served alone by the batched server
    strata = collections.defaultdict(list)
    for r in base:
        strata[(_schedule_class(r.n, r.kind), r.kind)].append(r)
    per = max(1, sample // max(1, len(strata)))
    picked = [r for v in strata.values() for r in v[:per]]
    srv = Server(budget_bytes, nstreams)
    errs = collections.defaultdict(list)
    import concurrent.futures as cf
    with cf.ThreadPoolExecutor(max_workers=8) as ex:
        jobs = []
        for r in picked:
            # the request's first transform, served alone into its own buffer
            xin = pools.input(r)[0]
            out = torch.empty(r.n, dtype=xin.dtype, device="cuda")
            tkt = ctypes.c_int64()
            _check(_lib.lib.fb_server_submit(srv.h, r.n, Server.KIND[r.kind], r.dir, 1,
                                             ctypes.c_void_p(xin.data_ptr()),
                                             ctypes.c_void_p(out.data_ptr()), ctypes.byref(tkt)))
            _check(_lib.lib.fb_server_wait(srv.h))
            x = xin.cpu().numpy().astype(np.complex128)
            jobs.append((r, out.cpu().numpy(), ex.submit(reference, x[None, :], r.dir)))
        for r, y, fut in jobs:
            ref = fut.result()[0]
            e = float(np.linalg.norm(y - ref) / np.linalg.norm(ref))
            errs[(_schedule_class(r.n, r.kind), r.kind)].append(e)
    del srv
    acc = {}
    for (cls, kind), v in sorted(errs.items()):
        acc[f"{kind}/{cls}"] = {"requests": len(v), "max_rel_l2": max(v),
                                "median_rel_l2": float(np.median(v))}
    result["accuracy_vs_fp64_oracle"] = acc
    result["max_rel_l2"] = {k: max(max(v) for (c, kk), v in errs.items() if kk == k)
                            for k in ("c64", "c128") if any(kk == k for (_, kk) in errs)}
    return result
