"""Generate fb_fast_table.inc: the lengths with compile-time kernels.

Each entry's radix list is the planner's radix program for that length
(fb_plan.cu radix_program: radix 16 with a trailing 8*4 / 4 / 8 / 2 for powers
of two, radix 9 with a trailing 3 for powers of three, then 5s and odd primes)
for the lengths below (powers of two and three, 2^a*3, 2^a*9, 5-smooth 5^c*2^a)
and T = L / (largest radix) threads per line (at most 512; 1024 from 16384 up
and where L / (largest radix) exceeds 512).
Entries are spread over PARTS compilation units so they build in parallel.

Run:  python gen_fast_table.py   (rewrites fb_fast_table.inc next to it)
"""
import os

PARTS = 4


def radix_program(L):
    r = []
    a = 0
    while L % 2 == 0:
        L //= 2
        a += 1
    q, rem = divmod(a, 4)
    if rem == 1 and q >= 1:
        r += [16] * (q - 1) + [8, 4]
    else:
        r += [16] * q + {0: [], 1: [2], 2: [4], 3: [8]}[rem]
    b = 0
    while L % 3 == 0:
        L //= 3
        b += 1
    r += [9] * (b // 2) + ([3] if b % 2 else [])
    p = 5
    while L > 1:
        while L % p == 0:
            r.append(p)
            L //= p
        p += 2
    return r


def lengths():
    out = set()
    for a in range(1, 15):
        out.add(2 ** a)
    for b in range(1, 9):
        out.add(3 ** b)
    for a in range(4, 13):
        out.add(2 ** a * 3)
        out.add(2 ** a * 9)
    # 5-smooth lengths (2-D and four-step factors such as 1000 = 25 x 40)
    for c in (2, 3, 4):
        for a in range(0, 6):
            out.add(5 ** c * 2 ** a)
    out.add(40)
    out.add(1000)
    out = {x for x in out if x <= 16384}
    # ComplexF32 lines beyond the generic kernel's limit that still fit one
    # SM's shared memory (1024 threads per line)
    out.add(3 ** 9)
    return sorted(out)


def main():
    lines = ["// Generated by gen_fast_table.py -- do not edit by hand.",
             "// FB_E(length, threads per line, radices...)"]
    ents = []
    for L in lengths():
        rad = radix_program(L)
        T = L // max(rad)
        if L == 16384 or (T > 512 and max(rad) == 16):
            # more radix-16 butterflies per stage than 512 threads: one per
            # thread on 1024 threads (16 values each, 64 registers, one block
            # per SM) rather than two per thread on 512 (32 values, 128
            # registers, one block of half the warps): the 9216-point
            # Bluestein pad of 2^8 * 4099 x 4 went from 0.240 to 0.214 ms.
            # Radix-8/9 programs (5000, 6561) measured within a few percent
            # either way and keep 512.
            T = 1024
        T = min(T, 1024 if L >= 16384 or T == 1024 else 512)
        wide = L * 16 > 8192 * 16  # longer than the ComplexF64 line limit
        ents.append((L, T, rad, wide))
    for part in range(PARTS):
        lines.append(f"#if FB_PART == {part}")
        for i, (L, T, rad, wide) in enumerate(ents):
            if i % PARTS != part:
                continue
            e = f"    FB_E({L}, {T}, {', '.join(map(str, rad))}),"
            lines.append(f"#if FB_WIDE_LINES\n{e}\n#endif" if wide else e)
        lines.append("#endif")
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "fb_fast_table.inc"), "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
