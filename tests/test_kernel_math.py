"""CPU checks of the arithmetic two kernels rely on, restated in Python on
small seeded cases (the kernels themselves are checked on the GPU).

k_crt_lin (ffg_crt.cu): a doubling step's outputs alpha s1 + beta s2 + gamma
formed per coefficient as Z_i = alpha X1_i + beta X2_i + K (2^b - 1),
K = 2^(94 - b), summed over the coefficients the CTAs cover, plus the
constant gamma + K, equal the outputs modulo 2^(64 len); every Z_i lies in
[0, 2^96).

k_school_sq_pair (ffg_crt.cu): column j of a square as 2 sum_{i < j - i}
a_i a_(j-i) + a_(j/2)^2, the pair sum split over 4 threads (i = part mod 4)
and combined in 192 bits, gives the square."""
import random

P3 = 2113929217 * 2013265921 * 1811939329
M64 = (1 << 64) - 1


def digits(x, w, n):
    return [(x >> (w * i)) & ((1 << w) - 1) for i in range(n)]


def convolution(a, b):
    out = [0] * (len(a) + len(b) - 1)
    for i, u in enumerate(a):
        if u:
            for j, v in enumerate(b):
                out[i + j] += u * v
    return out


def test_crt_lin_bias():
    rng = random.Random(1)
    for _ in range(120):
        w = rng.choice([32, 33, 34, 35])
        nk = rng.randint(1, 10)
        fk = rng.getrandbits(64 * nk) | (1 << (64 * nk - 1))
        fkm1 = rng.randrange(1, fk) >> rng.randint(0, 40)
        ca1, ca2 = (fk.bit_length() + w - 1) // w, (max(1, fkm1.bit_length()) + w - 1) // w
        X1 = convolution(digits(fk, w, ca1), digits(fk, w, ca1))
        X2 = convolution(digits(fkm1, w, ca2), digits(fkm1, w, ca2))
        assert max(X1) < P3
        s1, s2 = fk * fk, fkm1 * fkm1
        length = 2 * nk + 2
        NL = 32 * w                       # limbs per CTA
        ncta = (length + NL - 1) // NL
        covered = ncta * 2048             # coefficients the CTAs cover
        K = 1 << (94 - w)
        bias = K * ((1 << w) - 1)
        for al, be, ga in ((3, -2, 2), (4, -1, -2), (1, 1, 0), (3, -2, -2)):
            total = 0
            for i in range(covered):
                z = al * (X1[i] if i < len(X1) else 0) + be * (X2[i] if i < len(X2) else 0) + bias
                assert 0 <= z < 1 << 96
                total += z << (w * i)
            total += (ga + K) % (1 << 64)
            want = al * s1 + be * s2 + ga
            assert 0 <= want < 1 << (64 * length)
            assert total % (1 << (64 * length)) == want


def square_column(a, j, tpc=4):
    n = len(a)
    parts = []
    for part in range(tpc):
        t0 = t1 = t2 = 0
        if 1 <= j <= 2 * n - 3:
            for i in range(max(0, j - n + 1) + part, (j - 1) // 2 + 1, tpc):
                pr = a[i] * a[j - i]
                lo, hi = pr & M64, pr >> 64
                t0 = (t0 + lo) & M64
                h = hi + (1 if t0 < lo else 0)
                t1 = (t1 + h) & M64
                t2 += 1 if t1 < h else 0
        parts.append((t0, t1, t2))
    t0 = t1 = t2 = 0
    for q0, q1, q2 in parts:
        t0 = (t0 + q0) & M64
        c0 = 1 if t0 < q0 else 0
        x1 = (q1 + c0) & M64
        c1 = 1 if x1 < c0 else 0
        t1 = (t1 + x1) & M64
        t2 += q2 + c1 + (1 if t1 < x1 else 0)
    t2, t1, t0 = (t2 << 1) | (t1 >> 63), ((t1 << 1) & M64) | (t0 >> 63), (t0 << 1) & M64
    if 0 <= j <= 2 * n - 2 and j % 2 == 0:
        sq = a[j // 2] ** 2
        lo, hi = sq & M64, sq >> 64
        t0 = (t0 + lo) & M64
        c0 = 1 if t0 < lo else 0
        x1 = (hi + c0) & M64
        c1 = 1 if x1 < c0 else 0
        t1 = (t1 + x1) & M64
        t2 += c1 + (1 if t1 < x1 else 0)
    return t0 + (t1 << 64) + (t2 << 128)


def test_school_square_columns():
    rng = random.Random(3)
    for _ in range(40):
        n = rng.randint(1, 60)
        a = [rng.getrandbits(64) if rng.random() < 0.8 else M64 for _ in range(n)]
        x = sum(v << (64 * i) for i, v in enumerate(a))
        assert sum(square_column(a, j) << (64 * j) for j in range(2 * n + 1)) == x * x
