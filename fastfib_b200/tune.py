"""Autotuner of the multiply dispatch, and trainer of its learned cost model.

The reference picks its multiply by fixed thresholds (src/mul_basic.c:30-38)
and its transform length by the smallest 2^k or 3 2^(k-2) that fits
(src/mul_ntt.c:78-93).  Here the choice is measured: for sampled operand
shapes every candidate method (schoolbook, the reference's NTT plan, the
length forced to 2^k, forced to 3 2^k) is timed on the GPU inside a batch of
identical products (ffg_time_batch, device time per product), and an FP32
MLP (trained by the library's own CUDA kernels) learns log2 microseconds per
product from the shape features.  Method "learned" then takes, per product,
the candidate of least predicted cost; every candidate computes the exact
product, so the choice never changes a result.

The four-step geometry (row length, column-tile width) is tuned first, per
transform length, on pairs of squarings as the fast-doubling chain runs
them; the method timings and the cost model follow on that geometry.  Both
go to one text file that ffg_load_tuning reads (C hosts included):

    python -m fastfib_b200.tune --out fastfib_b200/tuning.txt
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

import fastfib_b200 as ff

SCHOOL_CAP = 1 << 27  # schoolbook candidates up to this many limb products (na * nb)


def sample_shapes(seed: int = 11, count: int = 320, lo: int = 10, hi: int = 24, max_aspect: int = 16,
                  square_frac: float = 0.2):
    """(bits_a, bits_b, square) drawn like the uneven product stream: bit
    lengths log-uniform over [2^lo, 2^hi], aspect at most max_aspect."""
    rng = np.random.default_rng(seed)
    span = math.log2(max_aspect)
    out = []
    for _ in range(count):
        la = rng.uniform(lo, hi)
        sq = rng.random() < square_frac
        lb = la if sq else rng.uniform(max(lo, la - span), min(hi, la + span))
        out.append((int(2 ** la), int(2 ** lb), bool(sq)))
    return out


def _torch():
    import torch
    return torch


def time_shape(bits_a: int, bits_b: int, square: bool, method: str, budget_limbs: int = 1 << 23,
               reps: int = 3, k: int = 0) -> float:
    """Device microseconds per product of `method` on a batch of k identical
    products of these bit lengths (random limbs; k = 0: from the budget)."""
    torch = _torch()
    na, nb = max(1, (bits_a + 63) // 64), max(1, (bits_b + 63) // 64)
    if square:
        nb, bits_b = na, bits_a
    if not k:
        k = int(min(512, max(1, budget_limbs // (na + nb))))
    if method == "school":
        k = int(min(k, max(1, (1 << 30) // (na * nb))))
    dev = torch.device("cuda:0")
    a = torch.randint(-2**63, 2**63 - 1, (k, na), dtype=torch.int64, device=dev)
    b = a if square else torch.randint(-2**63, 2**63 - 1, (k, nb), dtype=torch.int64, device=dev)
    out = torch.empty((k, na + nb + 1), dtype=torch.int64, device=dev)
    jobs = [{"a": a[i].data_ptr(), "b": None if square else b[i].data_ptr(), "na": na, "nb": nb,
             "bits_a": 64 * na, "bits_b": 64 * nb, "out": out[i].data_ptr(), "square": square, "method": method}
            for i in range(k)]
    ms = ff.time_batch(jobs, reps)
    del a, b, out
    return ms * 1000.0 / k


def collect(shapes, reps: int = 3, log=None):
    """Training rows: features, method index, log2 us per product."""
    X, M, Y, raw = [], [], [], []
    for s, (ba, bb, sq) in enumerate(shapes):
        na, nb = (ba + 63) // 64, (bb + 63) // 64
        f = ff.mlp_features(ba, ba if sq else bb, sq)
        for mi, name in enumerate(ff.MODEL_METHODS):
            if name == "school" and na * nb > SCHOOL_CAP:
                continue
            us = time_shape(ba, bb, sq, name, reps=reps)
            X.append(f)
            M.append(mi)
            Y.append(math.log2(us))
            raw.append((ba, bb, sq, name, us))
        if log and (s + 1) % 32 == 0:
            log(f"timed {s + 1}/{len(shapes)} shapes")
    return np.array(X, np.float32), np.array(M, np.int32), np.array(Y, np.float32), raw


def tune_geometry(lg_lo: int = 10, lg_hi: int = 24, reps: int = 5, log=None):
    """Per transform length (2^lg and 3 2^lg from 1024; up to 4096 against
    the one-CTA kernel, the default there) the fastest (row_lg, wc) on two
    squarings of about 0.9 L coefficients at a time, the fast-doubling
    chain's pair (device time of graph replays).  Returns the rows installed."""
    table = []
    cap = ff.ntt_max_L()
    for lg in range(lg_lo, lg_hi + 1):
        for r3 in (0, 1):
            L = (3 if r3 else 1) << lg
            if L < 1024 or L > cap:  # up to 4096 the default is the one-CTA transform
                continue
            bits = int(0.9 * L * 32 / 2)
            method = "ntt_r3" if r3 else "ntt_pow2"
            k = 2
            r = reps if L >= 1 << 16 else 4 * reps
            best = None
            for c in range(4, 14):
                for wc in (8, 16, 32, 64):
                    try:
                        ff.set_geometry(lg, r3, c, wc)
                    except ff.FfgError:
                        continue
                    us = time_shape(bits, bits, True, method, reps=r, k=k)
                    if best is None or us < best[0]:
                        best = (us, c, wc)
            ff.set_geometry(lg, r3, 0, 0)
            default = time_shape(bits, bits, True, method, reps=r, k=k)
            if best and best[0] < default:
                ff.set_geometry(lg, r3, best[1], best[2])
                table.append((lg, r3, best[1], best[2]))
            if log:
                log(f"L = {L}: default {default:.1f} us, best {best[0]:.1f} us at row_lg {best[1]} wc {best[2]}")
    return table


def choice_gain_bound(raw) -> float:
    """The most any per-product choice among the timed candidates could gain
    over the reference's thresholds on the sampled shapes: sum over shapes of
    the plain method's time over the sum of each shape's fastest candidate
    (schoolbook below a short side of 200 limbs, the NTT plan from there, as
    the reference's dispatch, src/mul_basic.c:30-38)."""
    by = {}
    for ba, bb, sq, name, us in raw:
        by.setdefault((ba, bb, sq), {})[name] = us
    plain = best = 0.0
    for (ba, bb, sq), t in by.items():
        short = min((ba + 63) // 64, (bb + 63) // 64)
        p = t["ntt"] if short >= 200 or "school" not in t else t["school"]
        plain += p
        best += min(t.values())
    return plain / best if best else 1.0


def fit(X, M, Y, epochs: int = 2000, lr: float = 1e-2, seed: int = 0):
    params, hist = ff.mlp_train(ff.mlp_init(seed), X, M, Y, epochs=epochs, lr=lr)
    return params, hist


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--shapes", type=int, default=320)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--epochs", type=int, default=2000)
    ap.add_argument("--lr", type=float, default=1e-2)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--no-geometry", action="store_true", help="keep the default four-step geometry")
    ap.add_argument("--out", default=ff.TUNING_PATH)
    ap.add_argument("--data", default="", help="also save the timing rows (npz)")
    args = ap.parse_args(argv)
    ff.init(1 << 24)  # tables to 2^25: geometry for every length up to 2^24 (and 3 2^23)
    t0 = time.time()
    geometry = [] if args.no_geometry else tune_geometry(log=print)
    t1 = time.time()
    shapes = sample_shapes(args.seed, args.shapes)
    X, M, Y, raw = collect(shapes, args.reps, log=print)
    t2 = time.time()
    params, hist = fit(X, M, Y, args.epochs, args.lr)
    pred = ff.mlp_predict(params, X)[np.arange(len(M)), M]
    rms = float(np.sqrt(np.mean((pred - Y) ** 2)))
    meta = {"rows": int(len(Y)), "shapes": args.shapes, "seed": args.seed, "epochs": args.epochs, "lr": args.lr,
            "loss_first": float(hist[0]), "loss_last": float(hist[-1]), "rms_log2_error": rms,
            "geometry_rows": len(geometry), "choice_gain_bound": round(choice_gain_bound(raw), 4),
            "geometry_s": round(t1 - t0, 1), "collect_s": round(t2 - t1, 1),
            "train_s": round(time.time() - t2, 1)}
    try:
        import torch
        meta["device"] = torch.cuda.get_device_name(0)
    except Exception:
        pass
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    ff.write_tuning(args.out, geometry, params, comment=json.dumps(meta))
    if args.data:
        shapes_arr = np.array([(r[0], r[1], r[2], ff.MODEL_METHODS.index(r[3])) for r in raw], dtype=np.int64)
        np.savez(args.data, params=params, X=X, M=M, Y=Y, shapes=shapes_arr, meta=json.dumps(meta))
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
