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


def settle(out, cta_limbs, maps, walk=8, long_max=64):
    """settle_cta (ffg_ripple.cuh) restated: the carry into every CTA from the
    composed maps; a CTA with the identity map zeroed outright, any other
    carried into by a bounded walk of `walk` limbs; carries
    still running go to a list finished 'by the block' (first limb that is
    not 2^64 - 1 gains 1, the ones before it become 0); past `long_max`
    entries the walk simply continues."""
    ncta = len(maps)
    carry, pending = 0, []
    for q in range(ncta):
        if carry and maps[q] == 2:  # the identity map: every limb 2^64 - 1, all wrap to 0
            for j in range(q * cta_limbs, min(len(out), (q + 1) * cta_limbs)):
                out[j] = 0
        elif carry:
            j, end = q * cta_limbs, min(len(out), (q + 1) * cta_limbs)
            running = True
            for _ in range(walk):
                if j >= end:
                    break
                out[j] = (out[j] + 1) & M64
                j += 1
                if out[j - 1] != 0:
                    running = False
                    break
            if running and j < end:
                if len(pending) < long_max:
                    pending.append((j, end))
                else:
                    while j < end:
                        out[j] = (out[j] + 1) & M64
                        j += 1
                        if out[j - 1] != 0:
                            break
        carry = (maps[q] >> carry) & 1  # bit c: carry out for carry in c
    for j0, end in pending:
        first = next((j for j in range(j0, end) if out[j] != M64), None)
        for j in range(j0, end if first is None else first):
            out[j] = 0
        if first is not None:
            out[first] += 1


def test_settle_long_carries():
    rng = random.Random(7)
    for trial in range(300):
        cta, ncta = rng.choice([4, 8, 32]), rng.randint(1, 12)
        n = cta * ncta - rng.randint(0, cta - 1)
        # per-CTA limbs as each CTA leaves them (no carry in), with runs of 2^64 - 1
        limbs = []
        for _ in range(n):
            r = rng.random()
            limbs.append(M64 if r < 0.8 else (0 if r < 0.83 else rng.getrandbits(64)))
        # a CTA's own carry out (c_in = 0); a CTA whose limbs all propagate
        # (2^64 - 1) generates none: a group's generate and propagate exclude each other
        carries_out = []
        for q in range(ncta):
            seg = limbs[q * cta:min(n, (q + 1) * cta)]
            carries_out.append(rng.random() < 0.5 and not all(v == M64 for v in seg))
        # the true value: each CTA's limbs plus its own carry out at the next CTA's start
        want = sum(v << (64 * i) for i, v in enumerate(limbs))
        for q in range(ncta - 1):
            if carries_out[q]:
                want += 1 << (64 * (q + 1) * cta)
        want &= (1 << (64 * n)) - 1
        # maps: carry out for c_in = 0 and 1 (c_in = 1 wraps the CTA when every limb is 2^64 - 1)
        maps = []
        for q in range(ncta):
            seg = limbs[q * cta:min(n, (q + 1) * cta)]
            all_ones = all(v == M64 for v in seg)
            c0 = int(carries_out[q])
            c1 = 1 if (c0 or all_ones) else 0
            maps.append(c0 | (c1 << 1))
        out = list(limbs)
        settle(out, cta, maps, walk=rng.choice([1, 2, 8]), long_max=rng.choice([1, 64]))
        assert sum(v << (64 * i) for i, v in enumerate(out)) == want, trial


def test_fingerprint_runs():
    """k_fp_partial (ffg_fingerprint.cu) restated: thread t reduces limbs
    [t*per, (t+1)*per) by Horner's rule from the top with 2^64 mod p, weights
    the run by (2^64)^(first limb) mod p, and the runs' residues sum to
    x mod p; runs past the end are empty."""
    primes = (18446744073709551557, 18446744073709551533, 9223372036854775783, 4611686018427387847)
    rng = random.Random(5)
    for n in (0, 1, 2, 7, 64, 1000, 4097):
        limbs = [rng.getrandbits(64) if rng.random() < 0.9 else M64 for _ in range(n)]
        x = sum(v << (64 * i) for i, v in enumerate(limbs))
        for nthreads in (1, 3, 256, 5000):
            per = (n + nthreads - 1) // nthreads
            for p in primes:
                r64 = (1 << 64) % p
                total = 0
                for t in range(nthreads):
                    i0, i1 = min(t * per, n), min(t * per + per, n)
                    h = 0
                    for i in range(i1 - 1, i0 - 1, -1):
                        h = (h * r64 + limbs[i]) % p
                    if h:
                        h = h * pow(r64, i0, p) % p
                    total = (total + h) % p
                assert total == x % p, (n, nthreads, p)


def _dif(x, p, w32, nz=None):
    """The in-register radix-2^M decimation in frequency of ffg_lines.cuh
    (dft_dif), or with nz set its pruned form for inputs zero at slots >= nz
    (dft_dif_nz): while the half distance h >= nz a pair (a, 0) becomes
    (a, a w) and all-zero pairs are skipped."""
    x = list(x)
    n = len(x)
    M = n.bit_length() - 1
    for lev in range(M):
        h = 1 << (M - 1 - lev)
        for t in range(n):
            if t & h:
                continue
            e = (t & (h - 1)) * (16 // h)
            w = pow(w32, e, p)
            if nz is not None and h >= nz:
                if (t & (h - 1)) >= nz:
                    continue
                x[t + h] = x[t] * w % p
            else:
                a, b = x[t], x[t + h]
                x[t], x[t + h] = (a + b) % p, (a - b) * w % p
    return x


def test_pruned_dif_matches_full():
    """The first column step's zero-row pruning (ffg_cols.cu col_fwd2_first,
    dft_dif_nz): for every radix 2..32 and every power-of-two count of
    nonzero leading slots, the pruned transform equals the full one."""
    rng = random.Random(5)
    for p, g in ((2113929217, 5), (2013265921, 31), (1811939329, 13)):
        w32 = pow(g, (p - 1) // 32, p)
        for M in range(1, 6):
            n = 1 << M
            for k in range(M + 1):
                nz = 1 << k
                for _ in range(20):
                    x = [rng.randrange(p) if t < nz else 0 for t in range(n)]
                    assert _dif(x, p, w32, nz) == _dif(x, p, w32)


# ---------------------------------------------------------------- addressing
# The fixed-shape passes (ffg_rows.cu, ffg_cols.cu) address shared memory
# with compile-time offsets from per-group bases.  Restated here for every
# shape they instantiate: each step touches every word of a line exactly
# once, stays inside its line, and a warp's simultaneous accesses fall in
# distinct banks.

COL_SHAPES = {6: (0, 1), 7: (0, 2), 8: (0, 3), 9: (0, 4), 10: (2, 3), 11: (3, 3), 12: (4, 3), 13: (4, 4)}
ROW_SHAPES = {9: (0, 4), 10: (0, 5), 11: (3, 3), 12: (4, 3), 13: (4, 4)}


def pad(i):
    return i + i // 32


def col2_stride(R, wc):
    wl = min(wc, 32)
    return ((R + R // 32 + 31) & ~31) + 32 // wl


def _col_steps(rn, r3):
    """(positions of each group) for steps A, B, C of one column line."""
    MA, MB = COL_SHAPES[rn]
    R, nblk = 1 << rn, 3 if r3 else 1
    BP = R + R // 32
    steps = []
    if MA:
        SA = R >> MA
        groups = []
        for q in range(nblk):
            for j in range(SA):
                groups.append([q * BP + j + j // 32 + t * (SA + SA // 32) for t in range(1 << MA)])
        steps.append(groups)
    NB = 32 << MB
    groups = []
    for b in range(nblk * R // NB):
        for j in range(32):
            groups.append([b * (NB + NB // 32) + j + 33 * t for t in range(1 << MB)])
    steps.append(groups)
    groups = []
    for b in range(nblk * R // 32):
        q, bl = b >> (rn - 5), b & ((R >> 5) - 1)
        groups.append([q * BP + 33 * bl + t for t in range(32)])
    steps.append(groups)
    return steps


def test_column_pass_addressing():
    for rn in COL_SHAPES:
        for r3 in (False, True):
            if r3 and rn > 12:
                continue
            R = (3 if r3 else 1) << rn
            want = sorted(pad(i) for i in range(R))
            for groups in _col_steps(rn, r3):
                got = sorted(a for g in groups for a in g)
                assert got == want, (rn, r3)
            for wc in (8, 16, 32, 64):
                LS = col2_stride(R, wc)
                assert LS > pad(R - 1)
                # step C: lanes = (column s mod wc, group s / wc); same t
                C = _col_steps(rn, r3)[-1]
                for w0 in range(0, min(wc * len(C), 256), 32):
                    banks = set()
                    for s in range(w0, w0 + 32):
                        c, b = s % wc, s // wc
                        if b < len(C):
                            banks.add((c * LS + C[b][0]) % 32)
                    assert len(banks) == min(32, wc * len(C) - w0), (rn, r3, wc)


def test_row_pass_addressing():
    for clg, (MA, MB) in ROW_SHAPES.items():
        C = 1 << clg
        T = C // 32
        want = sorted(pad(i) for i in range(C))
        seen_a = []
        if MA:
            SA = C >> MA
            for tau in range(T):
                for k in range(32 >> MA):
                    j = tau + T * k
                    seen_a += [j + j // 32 + t * (SA + SA // 32) for t in range(1 << MA)]
            assert sorted(seen_a) == want
        NB = 32 << MB
        seen_b = []
        for tau in range(T):
            for k in range(32 >> MB):
                g = tau + T * k
                b, j = g >> 5, g & 31
                seen_b += [b * (NB + NB // 32) + j + 33 * t for t in range(1 << MB)]
        assert sorted(seen_b) == want
        assert sorted(33 * tau + t for tau in range(T) for t in range(32)) == want
