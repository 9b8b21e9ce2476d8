"""Generate tests/golden/dft_golden.npz: 50-digit DFTs of seeded inputs.

Independent of both the CPU oracle and the CUDA library: each output is the
direct sum X_k = sum_n x_n exp(-2 pi i n k / N) (forward) or with +i
(backward) evaluated with mpmath at 50 significant digits, then rounded to
complex128.  The lengths cover every schedule class of the reference's call
graph (FFTA src/callgraph.jl:86-125): N=1, powers of 2 and 3, primes below
the Bluestein cutoff 73 (DFT leaves), primes at or above it (Bluestein), and
composites whose split takes the `N_cp[idx+1]` branch (275) or nests
composites (100, 1000 is left to the oracle).  Inputs are complex normal
from numpy's PCG64 with the seed stored next to each case.

Run:  python tests/golden/make_golden.py
"""
import os

import mpmath
import numpy as np

mpmath.mp.dps = 50
SIZES = [1, 2, 3, 4, 5, 6, 7, 8, 9, 11, 12, 13, 15, 16, 17, 25, 27, 30, 31, 32, 45, 49, 64,
         71, 73, 81, 97, 100, 103, 128, 210, 243, 256, 275, 289]


def dft(x, sign):
    n = len(x)
    xs = [mpmath.mpc(complex(v)) for v in x]
    out = np.empty(n, dtype=np.complex128)
    for k in range(n):
        s = mpmath.mpc(0)
        for j in range(n):
            s += xs[j] * mpmath.expjpi(sign * mpmath.mpf(2 * ((j * k) % n)) / n)
        out[k] = complex(s)
    return out


def main():
    data = {}
    for n in SIZES:
        seed = 1000 + n
        rng = np.random.default_rng(seed)
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        data[f"x_{n}"] = x
        data[f"fwd_{n}"] = dft(x, -1)
        data[f"bwd_{n}"] = dft(x, +1)
        data[f"seed_{n}"] = np.array(seed)
    data["sizes"] = np.array(SIZES)
    here = os.path.dirname(os.path.abspath(__file__))
    np.savez_compressed(os.path.join(here, "dft_golden.npz"), **data)


if __name__ == "__main__":
    main()
