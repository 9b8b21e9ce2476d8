"""Autotuner (fb_plan_autotune, fb_tune_cache_save/load).

FFTA has no tuner (its plans are fixed by src/callgraph.jl:76-126); the
tuner here only chooses launch shapes, so every GPU test checks that the
transform's result is unchanged bit for bit after tuning.
"""
import numpy as np
import pytest

import ffta_b200 as F


def test_cache_file_round_trip(tmp_path):
    # a key no real plan has (type 9), so later plans are unaffected
    src = tmp_path / "in.txt"
    src.write_text("# comment\n9:-1:73:0:7/1/1,:0,|2,256,0;\n")
    F.load_tuning(str(src))
    out = tmp_path / "out.txt"
    F.save_tuning(str(out))
    lines = [l for l in out.read_text().splitlines() if not l.startswith("#")]
    assert "9:-1:73:0:7/1/1,:0,|2,256,0;" in lines


def test_cache_load_missing_file(tmp_path):
    with pytest.raises(F.ArgumentError, match="cannot read"):
        F.load_tuning(str(tmp_path / "absent.txt"))


def test_autotune_rejects_host_arrays():
    x = np.zeros(64, np.complex64)
    with pytest.raises(F.ArgumentError, match="device tensors"):
        F.autotune(F.plan_fft(x), x)


CASES = [
    ("c64", (4096, 512), 1),        # one fast direct pass
    ("c64", (1024, 1024), (1, 2)),  # direct + tile passes
    ("c64", (1 << 20,), 1),         # four-step
    ("c128", (5329, 16), 1),        # Bluestein
    ("c128", (1 << 16, 4), 1),      # four-step, ComplexF64
    ("c64", (12, 4096), 2),         # strided short lines
]


def _column_major(shape, dt, seed):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.randn(tuple(reversed(shape)), dtype=dt, device="cuda", generator=g)
    return x.permute(*reversed(range(len(shape))))


@pytest.mark.gpu
@pytest.mark.parametrize("kind,shape,region", CASES)
def test_autotune_keeps_results(kind, shape, region, tmp_path):
    import torch
    dt = torch.complex64 if kind == "c64" else torch.complex128
    x = _column_major(shape, dt, 7)
    p = F.plan_fft(x, region)
    before = (p * x).cpu()
    desc0 = p.describe(x)
    desc1 = F.autotune(p, x, iters=3)
    after = (p * x).cpu()
    assert torch.equal(before, after), (desc0, desc1)
    # a new plan of the same layout starts from the tuned shapes
    q = F.plan_fft(x, region)
    assert q.describe(x) == desc1
    assert torch.equal((q * x).cpu(), before)
    # the cache survives a save / load
    path = str(tmp_path / "tune.txt")
    F.save_tuning(path)
    F.load_tuning(path)
    assert F.plan_fft(x, region).describe(x) == desc1


@pytest.mark.gpu
def test_autotune_generic_only_plan():
    import torch
    x = _column_major((300, 2048), torch.complex64, 3)
    p = F.plan_fft(x, 1, _flags=F.FB_FLAG_GENERIC_ONLY)
    before = (p * x).cpu()
    F.autotune(p, x, iters=2)
    assert torch.equal((p * x).cpu(), before)


def _radices(desc):
    import re
    return re.findall(r"radices=([0-9x]+)", desc)


@pytest.mark.gpu
def test_radix_order_tuning():
    """FB_FLAG_TUNE_RADIX: the tuner also times alternative radix programs of
    each one-pass length (16/8/4/2 groupings of 2^a, 9/3 of 3^b, powers of
    two or of three first) and keeps the fastest, per (length, type,
    direction); later plans with the flag start from it.  A tuned plan is
    not bit-identical to the default one, so results are checked against the
    FP64 oracle within 4 eps log2 N.  Lengths without a specialised kernel
    (generic runtime programs) are where the order matters most."""
    import os
    import torch
    import oracle
    shapes = [((224, 512), "c64"), ((448, 256), "c64"), ((1792, 64), "c64"), ((352, 512), "c64"),
              ((2592, 64), "c64"), ((864, 128), "c128"), ((3584, 64), "c64"), ((4096, 256), "c64")]
    changed = []
    for shape, kind in shapes:
        dt = torch.complex64 if kind == "c64" else torch.complex128
        x = _column_major(shape, dt, shape[0])
        p = F.plan_fft(x, 1, _flags=F.FB_FLAG_TUNE_RADIX)
        d0 = p.describe(x)
        F.autotune(p, x, iters=5)
        d1 = p.describe(x)
        ref = oracle.fft_nd(x.cpu().numpy().astype(np.complex128), 1, -1, prec="f64",
                            nthreads=os.cpu_count() or 1)
        y = (p * x).cpu().numpy()
        eps = 2.0 ** -23 if kind == "c64" else 2.0 ** -52
        err = np.linalg.norm(y - ref) / np.linalg.norm(ref)
        assert err <= 4 * eps * np.log2(shape[0]), (shape, d1, err)
        if _radices(d0) != _radices(d1):
            changed.append((shape, _radices(d0), _radices(d1)))
            # a new plan with the flag starts from the tuned program
            q = F.plan_fft(x, 1, _flags=F.FB_FLAG_TUNE_RADIX)
            assert _radices(q.describe(x)) == _radices(d1)
            assert _radices(F.plan_fft(x, 1).describe(x)) == _radices(d0)  # default untouched
    assert changed, "the default program won for every length"
