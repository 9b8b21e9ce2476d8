"""Serving loop: trace generation (host) and, on the GPU, continuous batching.

The GPU tests check that every request's result is the same when it runs in
the mix (grouped launches, several streams, admission under a budget) as when
it runs alone, and that results match the oracle within the parity tolerance.
"""
import numpy as np
import pytest

from ffta_b200 import serving


def test_trace_distribution():
    tr = serving.make_trace(4000, rate=1000.0, seed=3)
    ns = np.array([r.n for r in tr])
    assert ns.min() >= 2 and ns.max() <= 2 ** 21
    pow2 = np.mean([(n & (n - 1)) == 0 for n in ns])
    assert 0.42 < pow2 < 0.58
    primes = np.mean([serving._is_prime(int(n)) for n in ns])
    assert 0.1 < primes < 0.2
    c64 = np.mean([r.kind == "c128" for r in tr])
    assert 0.15 < c64 < 0.25
    assert all(1 <= r.batch <= 512 for r in tr)
    arr = np.array([r.arrival for r in tr])
    assert np.all(np.diff(arr) >= 0)
    assert abs(len(tr) / arr[-1] - 1000.0) < 100.0


@pytest.mark.gpu
def test_mix_equals_alone_and_oracle():
    import torch
    import oracle
    tr = serving.make_trace(60, rate=2000.0, seed=5, n_max=2 ** 14, batch_max=8)
    xs = serving.make_inputs(tr, "cuda")
    ys = [torch.empty_like(x) for x in xs]
    cache = serving.PlanCache()
    serving.warm_plans(tr, cache)
    srv = serving.Server(budget_bytes=64 << 20, nstreams=3)
    st = srv.run(tr, xs, ys)
    assert st["requests"] == len(tr) and st["launches"] <= len(tr)
    assert serving.check_mix_equals_alone(tr, xs, ys, cache) == 0.0
    for r, x, y in list(zip(tr, xs, ys))[:20]:
        ref = oracle.fft_nd(x.cpu().numpy().T, 1, r.dir, prec="f64").T
        eps = 2.0 ** -23 if r.kind == "c64" else 2.0 ** -52
        err = np.linalg.norm(y.cpu().numpy() - ref) / np.linalg.norm(ref)
        assert err <= 4 * eps * max(1.0, np.log2(r.n)), (r, err)


@pytest.mark.gpu
def test_one_launch_for_mixed_requests():
    """Requests of different lengths, types and directions that are queued
    together go out as one descriptor launch per kernel variant, and each
    result equals the same transform run alone through its own plan."""
    import torch
    import ffta_b200 as F
    spec = [(4096, "c64", -1, 1), (1000, "c64", 1, 3), (4096, "c64", 1, 7), (243, "c64", -1, 2),
            (97, "c64", -1, 5), (2048, "c128", -1, 2), (35, "c128", 1, 4)]
    reqs = [serving.Request(i, n, k, d, b, i, 0.0) for i, (n, k, d, b) in enumerate(spec)]
    xs = serving.make_inputs(reqs, "cuda")
    ys = [torch.empty_like(x) for x in xs]
    st = serving.Server(nstreams=2).run(reqs, xs, ys)
    # one launch per (type, kernel variant, shared-memory class): 2 for C32, 2 for C64
    assert st["descriptor_launches"] <= 4 and st["launches"] == st["descriptor_launches"]
    for r, x, y in zip(reqs, xs, ys):
        f = F.fft if r.dir < 0 else F.bfft
        assert torch.equal(y, f(x.T, 1).T), r


@pytest.mark.gpu
def test_multipass_plans_share_stream_scratch():
    """Multi-pass requests of different schedules (four-step, three-pass
    Bluestein, a four-step with a Bluestein factor) and both types, all on
    one plan stream, so every plan uses that stream's shared scratch in turn;
    each is served twice in the same mix (the second time by a cached plan
    whose tables may come from the server's block cache).  Every result must
    equal the same transform run alone through its own plan, bit for bit."""
    import torch
    import ffta_b200 as F
    spec = [(20000, "c64", -1, 3), (100003, "c64", 1, 2), (3 * 2 ** 17, "c64", -1, 2),
            (30030, "c128", 1, 3), (65537, "c64", -1, 2), (2 ** 8 * 4099, "c64", 1, 1),
            (27648, "c128", -1, 2)]
    spec = spec + spec
    reqs = [serving.Request(i, n, k, d, b, i, 0.0) for i, (n, k, d, b) in enumerate(spec)]
    xs = serving.make_inputs(reqs, "cuda")
    ys = [torch.empty_like(x) for x in xs]
    st = serving.Server(nstreams=1, graphs=False).run(reqs, xs, ys)
    assert st["requests"] == len(reqs)
    for r, x, y in zip(reqs, xs, ys):
        f = F.fft if r.dir < 0 else F.bfft
        assert torch.equal(y, f(x.T, 1).T), (r.n, r.kind, r.dir, r.batch)


@pytest.mark.gpu
@pytest.mark.parametrize("graphs", [True, False])
def test_recurring_multipass_requests_replay_graphs(graphs):
    """Multi-pass requests (three-pass Bluestein, four-step) and large
    single-pass ones run through cached plans; when the same request recurs on
    the same buffers it is captured into a CUDA graph on its second occurrence
    and replayed from the third on.  Replayed results equal the plans' own
    launches bit for bit."""
    import torch
    import ffta_b200 as F
    spec = [(65537, "c64", -1, 1), (32768, "c64", 1, 2), (19683, "c128", 1, 1),
            (4096, "c64", -1, 64), (1000, "c64", 1, 3)]
    reqs = [serving.Request(i, n, k, d, b, i, 0.0) for i, (n, k, d, b) in enumerate(spec)]
    xs = serving.make_inputs(reqs, "cuda")
    ys = [torch.empty_like(x) for x in xs]
    srv = serving.Server(nstreams=2, graphs=graphs)
    plan_runs = 4  # every request but the packed 1000 x 3
    st = [srv.run(reqs, xs, ys)]
    for _ in range(2):
        for y in ys:
            y.fill_(float("nan"))
        st.append(srv.run(reqs, xs, ys))
    if graphs:
        assert [s["graph_captures"] for s in st] == [0, plan_runs, 0]
        assert [s["graph_launches"] for s in st] == [0, plan_runs, plan_runs]
    else:
        assert all(s["graph_captures"] == 0 and s["graph_launches"] == 0 for s in st)
    for r, x, y in zip(reqs, xs, ys):
        f = F.fft if r.dir < 0 else F.bfft
        assert torch.equal(y, f(x.T, 1).T), r


@pytest.mark.gpu
def test_graph_cache_releases_least_recently_used():
    """More recurring (plan, buffers) keys than the server keeps graphs for
    (1024): the least recently used graphs are released while later launches
    run, and every result still equals the plan's own launch."""
    import torch
    import ffta_b200 as F
    count = 1100
    reqs = [serving.Request(i, 20000, "c64", -1 if i % 2 else 1, 1, i, 0.0) for i in range(count)]
    base = torch.randn(count, 20000, dtype=torch.complex64, device="cuda")
    xs = [base[i:i + 1] for i in range(count)]
    ys = [torch.empty_like(x) for x in xs]
    srv = serving.Server(nstreams=2)
    st = [srv.run(reqs, xs, ys) for _ in range(3)]
    # run 2 captures every key (evicting the first 76 again); run 3 replays
    # the 1024 kept and sees the evicted ones for the first time since
    assert [s["graph_captures"] for s in st] == [0, count, 0]
    assert [s["graph_launches"] for s in st] == [0, count, 1024]
    fwd = F.fft(base.T, 1).T
    bwd = F.bfft(base.T, 1).T
    for i, y in enumerate(ys):
        assert torch.equal(y[0], (fwd if i % 2 else bwd)[i]), i


@pytest.mark.gpu
def test_resident_kernel_serves_small_requests():
    """Small requests of lengths 16..4096 (powers of two) go to the resident
    kernel: a persistent launch that claims chunks of queued work
    descriptors.  Each result equals the plan's own specialised kernel bit
    for bit and the FP64 oracle within tolerance; the kernel ends when idle
    and is launched again for later requests."""
    import time
    import torch
    import ffta_b200 as F
    import oracle
    rng = np.random.default_rng(21)
    spec = [(int(2 ** rng.integers(4, 13)), "c64" if rng.random() < 0.7 else "c128",
             -1 if rng.random() < 0.5 else 1, int(rng.integers(1, 40))) for _ in range(120)]
    reqs = [serving.Request(i, n, k, d, b, i, 0.0) for i, (n, k, d, b) in enumerate(spec)]
    xs = serving.make_inputs(reqs, "cuda")
    srv = serving.Server(nstreams=2)
    for rnd in range(2):
        ys = [torch.full_like(x, float("nan")) for x in xs]
        st = srv.run(reqs, xs, ys)
        assert st["resident_kernel_requests"] == len(reqs) and st["failed_requests"] == 0, st
        assert st["descriptor_launches"] == 0
        for r, x, y in zip(reqs, xs, ys):
            f = F.fft if r.dir < 0 else F.bfft
            assert torch.equal(y, f(x.T, 1).T), r
        for r, x, y in list(zip(reqs, xs, ys))[:12]:
            ref = oracle.fft_nd(x.cpu().numpy().T, 1, r.dir, prec="f64").T
            eps = 2.0 ** -23 if r.kind == "c64" else 2.0 ** -52
            err = np.linalg.norm(y.cpu().numpy() - ref) / np.linalg.norm(ref)
            assert err <= 4 * eps * max(1.0, np.log2(r.n)), (r, err)
        time.sleep(0.05)  # the kernel ends after 2 ms without work


@pytest.mark.gpu
def test_resident_kernel_gives_up_on_a_lost_descriptor():
    """A descriptor whose write is lost (fb_server_drop_next_descriptor): the
    resident kernel waits for it a bounded time, completes it with
    done_ms = -1 and serves the requests queued behind it."""
    import ctypes
    import torch
    import oracle
    from ffta_b200 import _lib
    h = ctypes.c_void_p()
    assert _lib.lib.fb_server_create(ctypes.byref(h), 8e9, 2, 0) == 0, _lib.last_error()
    try:
        g = torch.Generator(device="cuda").manual_seed(4)
        xs = [torch.randn(8, 1024, dtype=torch.complex64, device="cuda", generator=g)
              for _ in range(3)]
        ys = [torch.full_like(x, float("nan")) for x in xs]
        tk = ctypes.c_int64()
        tickets = []
        for i, (x, y) in enumerate(zip(xs, ys)):
            if i == 1:
                assert _lib.lib.fb_server_drop_next_descriptor(h) == 0
            assert _lib.lib.fb_server_submit(h, 1024, _lib.FB_C32, -1, 8,
                                             ctypes.c_void_p(x.data_ptr()),
                                             ctypes.c_void_p(y.data_ptr()),
                                             ctypes.byref(tk)) == 0, _lib.last_error()
            tickets.append(tk.value)
        assert _lib.lib.fb_server_wait(h) == 0, _lib.last_error()
        tks = (ctypes.c_int64 * 8)()
        tms = (ctypes.c_double * 8)()
        cnt = ctypes.c_int64()
        assert _lib.lib.fb_server_poll(h, 8, tks, tms, ctypes.byref(cnt)) == 0
        done = dict(zip(tks[:cnt.value], tms[:cnt.value]))
        assert sorted(done) == sorted(tickets)
        assert done[tickets[1]] == -1.0 and done[tickets[0]] >= 0 and done[tickets[2]] >= 0
        st = (ctypes.c_int64 * 11)()
        assert _lib.lib.fb_server_stats(h, st, 11) == 0
        assert st[9] == 3 and st[10] == 1
        torch.cuda.synchronize()
        assert torch.isnan(ys[1]).all()
        for i in (0, 2):
            ref = oracle.fft_batched(xs[i].cpu().numpy().astype(np.complex128), -1)
            err = np.linalg.norm(ys[i].cpu().numpy() - ref) / np.linalg.norm(ref)
            assert err <= 4 * 2.0 ** -23 * 10, err
    finally:
        _lib.lib.fb_server_destroy(h)


def test_output_ring_reuses_freed_space():
    """The configuration-5 driver's output ring (host logic): spans never
    overlap a live one, the ring wraps, and space frees on completion."""
    ring = serving._Ring(4096, device="cpu")
    a = ring.alloc(1500, 1)
    b = ring.alloc(1500, 2)
    assert (a, b) == (0, 1536)
    assert ring.alloc(1500, 3) is None  # 3072 + 1536 > 4096 and [0, 1536) is live
    ring.free(1)
    c = ring.alloc(1500, 3)  # wraps to the start
    assert c == 0
    spans = sorted((s0, ring.end[s0]) for s0 in ring.live.values())
    assert all(e1 <= s2 for (s1, e1), (s2, e2) in zip(spans, spans[1:]))
    with pytest.raises(ValueError):
        ring.alloc(5000, 4)
    r = serving.Request(0, 16, "c64", -1, 2, 0, 0.0)
    assert ring.view(c, r).shape == (2, 16)


def test_output_ring_random_against_brute_force():
    """Random allocations and out-of-order frees: the ring's answer equals a
    brute-force scan over the live spans (first fit at the head, else at 0)."""
    rng = np.random.default_rng(3)
    size = 1 << 16
    ring = serving._Ring(size, device="cpu")
    live, head = {}, 0
    for rid in range(3000):
        if live and rng.random() < 0.45:
            k = list(live)[rng.integers(len(live))]
            ring.free(k)
            live.pop(k)
            continue
        nb = int(rng.integers(1, 6000))
        rb = (nb + 255) // 256 * 256
        want = None
        for st in (head, 0):
            if st + rb <= size and all(e <= st or s0 >= st + rb for s0, e in live.values()):
                want = st
                break
        got = ring.alloc(nb, rid)
        assert got == want
        if got is not None:
            live[rid] = (got, got + rb)
            head = got + rb
