"""The bench's sweep over the size categories of FFTA's own benchmark suite
(benchmark/common_defs.jl): the host-side size list, checked on CPU."""
import importlib.util
import os


def _bench():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("bench_sizes_mod", os.path.join(root, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_reference_benchmark_sizes():
    cats = _bench().reference_benchmark_sizes()
    by = {}
    for n, c in cats.items():
        by.setdefault(c, []).append(n)
    # later categories overwrite earlier ones, as in create_size_categories():
    # 2 and 3 are listed as primes
    assert sorted(by["odd_power_of_2"]) == [2 ** i for i in range(3, 20, 2)]
    assert sorted(by["even_power_of_2"]) == [2 ** i for i in range(2, 21, 2)]
    assert sorted(by["power_of_3"]) == [3 ** i for i in range(2, 10)]
    assert sorted(by["composite"]) == [3, 12, 60, 300, 2100, 23100][1:]
    primes = sorted(by["prime"])
    assert primes[0] == 2 and primes[-1] <= 20000 and len(primes) == 20
    assert all(all(p % f for f in range(2, int(p ** 0.5) + 1)) for p in primes)
    assert len(cats) == 52 and max(cats) == 2 ** 20


def test_reference_arm_prints_the_contract_line():
    """`bench.py --impl reference` times FFTA's algorithm (the C++
    restatement) on the host cores and prints one JSON line on the headline's
    metric, with its e2e moving no bytes between host and device."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        env.pop(k, None)
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "1"], capture_output=True, text=True,
                         timeout=600, env=env, cwd=root)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "batched FFT GFLOP/s (5 N log2 N), C32 N=4096 x 16384"
    assert d["unit"] == "GFLOP/s" and d["higher_is_better"] is True and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "GFLOP/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
