#!/usr/bin/env python
"""Benchmark: F(n) in milliseconds on the B200 (default n = 10^8), bit-exact.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--n 100000000]
    python bench.py --impl reference ...     # the reference's CPU path

One step = one F(n) by fast doubling through the public API (fibonacci()).
`value` is the device time of the chain (CUDA events on the library's stream,
operands resident in HBM from the first doubling step on), `e2e` the same
call timed on the host including the prefix, the copy of the starting pair
to the device and the copy of F(n) back.  The roofline figures come from a
second pass of the same steps with CUDA events around every launch of the
dominant kernel family (kept out of the timed pass, which they perturb).  L2 is flushed (a 256 MiB write)
before every step.  With N > 1 every rank computes its own F(n) (replicas:
the chain is sequential and has no data-parallel split); value is the job's
ms per F(n), the max over ranks divided by N.  Prints one JSON line on rank 0.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.set_int_max_str_digits(0)

GOLD_FP = os.path.join(ROOT, "tests", "golden", "fingerprints.json")
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC = os.path.join(ROOT, "profiles", "roofline_traffic.json")
METRIC = "F(n) ms at n=1e8/1e9 on 1 B200, bit-exact; learned vs plain; NTT % HBM peak"
PUBLISHED_F1E8_MS = 46.0  # the reference's README, F(10^8) on an i9-9900K
# how oracle/_ref is compiled (oracle/Makefile): the reference's own sources,
# unmodified; it asks for -march=native, the AVX2 level it needs is x86-64-v3
REF_BUILD = "gcc -O3 -march=x86-64-v3 from the reference's sources (it asks for -march=native)"
FALLBACK_HBM_GBS = 6650.0  # an earlier copy-bandwidth measurement on B200


def hbm_peak():
    """(GB/s, source): the measured copy bandwidth from MEASURED_PEAKS.json
    when it is present, else the earlier measurement."""
    if os.path.exists(PEAKS):
        with open(PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return FALLBACK_HBM_GBS, "fallback (6.65 TB/s; MEASURED_PEAKS.json absent)"


def workload(n):
    return {"workload": f"F({n}) by fast doubling from (F(0), F(1)): 2 squarings + 1 linear pass per bit, "
                        f"last bit one product; three-prime NTT products on the device",
            "n": n, "l2": "flushed before every step (256 MiB write)", "parallelism": "replicas"}


def fingerprint_ok(n, limbs, device_fp=None):
    """F(n) against its committed fingerprint (bit length, low 64 bits, and the
    value mod four 64-bit primes, the format of the reference's memrun.c),
    computed with Python integers or by `device_fp` (the library's kernel)."""
    with open(GOLD_FP) as f:
        gold = json.load(f)
    want = gold["fingerprints"].get(str(n))
    if want is None:
        return None
    if device_fp is not None:
        return [str(v) for v in device_fp(limbs)] == want
    import numpy as np
    x = int.from_bytes(np.ascontiguousarray(limbs, dtype=np.uint64).tobytes(), "little")
    fp = [x.bit_length(), x & (2**64 - 1)] + [x % int(p) for p in gold["primes"]]
    return [str(v) for v in fp] == want


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(n, steps=7):
    """The reference's own CPU path on this host's cores (oracle/_ref), else our port."""
    from oracle import Oracle, Reference, reference_available
    if reference_available():
        ref, kind = Reference(), "reference"
        cores = ref.cpus()
        run = ref.fibonacci
    else:
        ref, kind, cores = Oracle(), "port", 1
        run = ref.fibonacci
    best = float("inf")
    run(n)
    for _ in range(steps):
        t = time.perf_counter()
        run(n)
        best = min(best, time.perf_counter() - t)
    out = {"value": best * 1e3, "unit": "ms", "cores": cores, "kind": kind,
           "sample": f"F({n}) best of {steps} runs after one warm-up, all pool threads"}
    if kind == "reference":
        out["build"] = REF_BUILD
    if kind == "reference":
        f = run(n)
        dec = float("inf")
        for _ in range(3):
            t = time.perf_counter()
            ref.to_string(f)
            dec = min(dec, time.perf_counter() - t)
        out["decimal_ms"] = dec * 1e3
        out["decimal_sample"] = f"big_to_string(F({n})) best of 3, all pool threads"
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    from oracle import Oracle, Reference, reference_available
    base = {"metric": METRIC, "impl": "reference", "unit": "ms", "higher_is_better": False, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "config": workload(args.n), "dtype": "u32",
            "data": "synthetic (F(n) needs no input data)"}
    if reference_available():
        lib, kind = Reference(), "reference"
        cores = lib.cpus()
    else:
        lib, kind, cores = Oracle(), "port", 1
    for _ in range(args.warmup):
        lib.fibonacci(args.n)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        r = lib.fibonacci(args.n)
        times.append((time.perf_counter() - t) * 1e3)
    v = statistics.mean(times)
    ok = fingerprint_ok(args.n, r)
    base.update({"value": v, "ms_per_step": v, "scaling": "weak", "vs_baseline": v / PUBLISHED_F1E8_MS
                 if args.n == 10**8 else None,
                 "cpu_baseline": {"value": v, "unit": "ms", "cores": cores, "kind": kind,
                                  "sample": f"F({args.n}) x {args.steps} after {args.warmup} warm-ups",
                                  **({"build": REF_BUILD} if kind == "reference" else {})},
                 "e2e": {"value": v, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                 "bit_exact": ok})
    print(json.dumps(base), flush=True)
    return 0


def run_ntt_microbench(args):
    line = ntt_microbench(args.limbs, args.square, args.steps, args.warmup)
    print(json.dumps(line), flush=True)
    return 0 if line["bit_exact"] else 1


def ntt_microbench(limbs, square, steps, warmup):
    """One NTT product of `limbs` random 64-bit limbs (seeded), square or
    distinct, repeated: per-family device times and each pass's fraction of
    the HBM roofline at that length (8 L bytes per prime per pass, twiddles
    excluded).  Operands stay on the device; L2 flushed before each step."""
    import numpy as np
    import torch
    import fastfib_b200 as ff
    torch.cuda.set_device(0)
    ff.set_device(0)
    ff.init(limbs * 2)
    rng = np.random.default_rng(88172645463325252 % 2**63)
    n = limbs
    a = rng.integers(0, 2**64, n, dtype=np.uint64)
    b = rng.integers(0, 2**64, n, dtype=np.uint64)
    a[-1] |= np.uint64(1 << 63)
    b[-1] |= np.uint64(1 << 63)
    da = torch.from_numpy(a.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    out = torch.zeros(2 * n + 1, dtype=torch.int64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    sq = square
    plan = ff.plan(64 * n, 64 * n, sq)

    def step():
        ff.mul_device(out.data_ptr(), da.data_ptr(), n, 64 * n, db.data_ptr(), n, 64 * n, sq)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    ff.profile(True)
    t_ms = []
    for i in range(steps):
        flush.fill_(i & 0xFF)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step()
        torch.cuda.synchronize()
        e1.record()
        torch.cuda.synchronize()
        t_ms.append(e0.elapsed_time(e1))
    prof = ff.profile_read()
    ff.profile(False)
    # check in O(n): the product modulo four 64-bit primes (exact products of
    # multi-million-limb integers in Python would take minutes)
    got = out.cpu().numpy().view(np.uint64)
    x, y = int.from_bytes(a.tobytes(), "little"), int.from_bytes(b.tobytes(), "little")
    z = int.from_bytes(got.tobytes(), "little")
    with open(GOLD_FP) as f:
        primes = [int(p) for p in json.load(f)["primes"]]
    ok = all(z % p == (x % p) * ((x if sq else y) % p) % p for p in primes) and z.bit_length() <= 128 * n
    peak, peak_src = hbm_peak()
    fam = {k: {"launches": v["launches"], "ms_per_launch": v["ms"] / max(1, v["launches"]),
               "gbs": v["bytes"] / (v["ms"] * 1e-3) / 1e9 if v["ms"] else 0.0,
               "frac": (v["bytes"] / (v["ms"] * 1e-3) / 1e9 / peak) if v["ms"] else 0.0}
           for k, v in prof.items() if v["launches"]}
    passes = [k for k in ("col_fwd", "row_conv", "col_inv") if k in fam]
    pb = sum(prof[k]["bytes"] for k in passes)
    pm = sum(prof[k]["ms"] for k in passes)
    return {"metric": "NTT multiply ms (microbench)", "value": statistics.mean(t_ms), "unit": "ms",
            "higher_is_better": False, "steps": steps, "warmup": warmup, "dtype": "u32",
            "config": {"workload": f"{'square' if sq else 'product'} of {n}-limb random operands", "plan": plan,
                       "l2": "flushed before every step"},
            "bit_exact": ok, "families": fam, "peak_gbs": peak,
            "ntt_passes": {"gbs": pb / (pm * 1e-3) / 1e9 if pm else 0.0,
                           "frac": (pb / (pm * 1e-3) / 1e9 / peak) if pm else 0.0,
                           "of": peak_src}}


def ntt_suite(steps=3, warmup=3, sizes=(1 << 14, 1 << 17, 1 << 20, 1 << 22), cpu=True):
    """The multiply microbench: random operands (seeded, uniform 64-bit limbs)
    of 2^14, 2^17, 2^20 and 2^22 limbs, squares and distinct products, each at
    the reference's own plan ("ntt") and with the transform length forced to
    2^k ("ntt_pow2") and to 3 2^k ("ntt_r3").  Device ms per product (CUDA
    events on the stream, L2 flushed before each, operands resident), every
    product checked modulo four 64-bit primes, and beside the plan's figure
    the reference's own big_mul / big_sqr on this host's cores (oracle/_ref,
    fastest of 3 calls, all pool threads)."""
    import numpy as np
    import torch
    import fastfib_b200 as ff
    torch.cuda.set_device(0)
    ff.set_device(0)
    ff.init(4 * max(sizes))  # tables up to 2^25: the forced 3 2^k lengths fit, no split
    ref = None
    if cpu:
        from oracle import Reference, reference_available
        ref = Reference() if reference_available() else None
    with open(GOLD_FP) as f:
        primes = [int(p) for p in json.load(f)["primes"]]
    rng = np.random.default_rng(88172645463325252 % 2**63)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    # a stream of our own: the library runs on the stream it is given, and the
    # events must be recorded on that same stream
    ts_stream = torch.cuda.Stream()
    stream = ts_stream.cuda_stream
    rows = []
    for n in sizes:
        a = rng.integers(0, 2**64, n, dtype=np.uint64)
        b = rng.integers(0, 2**64, n, dtype=np.uint64)
        a[-1] |= np.uint64(1 << 63)
        b[-1] |= np.uint64(1 << 63)
        da = torch.from_numpy(a.view(np.int64)).cuda()
        db = torch.from_numpy(b.view(np.int64)).cuda()
        out = torch.zeros(2 * n + 1, dtype=torch.int64, device="cuda")
        xa, xb = int.from_bytes(a.tobytes(), "little"), int.from_bytes(b.tobytes(), "little")
        for sq in (True, False):
            want = [(xa % p) * ((xa if sq else xb) % p) % p for p in primes]
            row = {"limbs": n, "square": sq}
            for m in ("ntt", "ntt_pow2", "ntt_r3"):
                job = [{"a": da.data_ptr(), "b": (da if sq else db).data_ptr(), "na": n, "nb": n, "bits_a": 64 * n,
                        "bits_b": 64 * n, "out": out.data_ptr(), "square": sq, "method": m}]
                for _ in range(warmup):
                    ff.mul_batch_device(job, stream)
                ts = []
                for i in range(steps):
                    flush.fill_(i & 0xFF)
                    torch.cuda.synchronize()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(ts_stream)
                    ff.mul_batch_device(job, stream)
                    e1.record(ts_stream)
                    torch.cuda.synchronize()
                    ts.append(e0.elapsed_time(e1))
                z = int.from_bytes(out.cpu().numpy().tobytes(), "little")
                ok = all(z % p == w for p, w in zip(primes, want))
                pl = ff.plan(64 * n, 64 * n, sq) if m == "ntt" else None
                row[m] = {"ms": statistics.mean(ts), "bit_exact": ok}
                if pl:
                    row["plan"] = {"width": pl["width"], "L": pl["L"], "split": pl["split"]}
            if ref is not None:
                row["cpu_reference_ms"] = ref.time_mul(a, None if sq else b, square=sq, reps=3) * 1e3
                row["speedup_vs_cpu"] = row["cpu_reference_ms"] / row["ntt"]["ms"]
            rows.append(row)
        del da, db, out
    return {"rows": rows, "cpu": {"kind": "reference" if ref else None, "cores": ref.cpus() if ref else None,
                                  "sample": "big_mul / big_sqr on the same operands, fastest of 3 calls, "
                                            "NTT tables built first"},
            "bit_exact": all(r[m]["bit_exact"] for r in rows for m in ("ntt", "ntt_pow2", "ntt_r3"))}


def job_ms(totals, steps, world, device="cuda"):
    """Replicas: each of `world` ranks ran `steps` chains in totals = [device
    ms, host ms]; the job's time is the max over ranks (an all-reduce MAX when
    world > 1), and per F(n) of the whole job it is that over steps * world."""
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor(list(totals), dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        totals = t.tolist()
    return [v / (steps * world) for v in totals]


def run_decimal(n=10**8, reps=3):
    """Decimal digits of F(n) through the device conversion (the reference's
    big_to_string, level by level with batched Barrett products): device ms
    of the levels and leaves (powers and reciprocals cached after the first
    call), wall ms of the host API call (number copied in, digits copied
    out), one call with the powers and reciprocals recomputed, and the digits
    against the reference's golden hash."""
    import hashlib
    import fastfib_b200 as ff
    f = ff.fibonacci(n)
    ff.to_decimal(f)  # the process's first conversion: arena growth, module loading
    ff.decimal_cache_clear()
    t = time.perf_counter()
    s, done = ff.to_decimal(f)  # powers and reciprocals recomputed, as the reference does every call
    first = (time.perf_counter() - t) * 1e3
    dev, wall = [], []
    for _ in range(reps):
        t = time.perf_counter()
        s, done = ff.to_decimal(f)
        wall.append((time.perf_counter() - t) * 1e3)
        dev.append(ff.last_decimal_ms())
    with open(os.path.join(ROOT, "tests", "golden", "decimal_sha256.json")) as fh:
        gold = json.load(fh)
    ok = bool(done) and str(n) in gold and hashlib.sha256(s.encode()).hexdigest() == gold[str(n)]
    # where the conversion's device time goes: one more call with every launch
    # bracketed by events, per kernel family (the decimal kernels of
    # ffg_decimal.cu count under "lin"; events perturb short launches)
    ff.profile(True)
    ff.to_decimal(f)
    fam = {k: {"launches": v["launches"], "ms": v["ms"]} for k, v in ff.profile_read().items() if v["launches"]}
    ff.profile(False)
    return {"n": n, "digits": len(s) if s else 0, "device_ms": statistics.median(dev),
            "e2e_ms": statistics.median(wall), "uncached_e2e_ms": first, "device_path": bool(done), "bit_exact": ok,
            "families": fam,
            "note": "device_ms / e2e_ms: powers of ten and reciprocals cached from an earlier call; "
                    "uncached_e2e_ms: recomputed inside the call, as the reference's big_to_string does"}


def run_uneven(count=4096, reps=3, seed=4):
    """The uneven product stream: `count` independent products, operand bit
    lengths log-uniform over 2^10..2^24, aspect up to 16:1, uniform random
    limbs (seeded), operands resident on the device.  Device ms of
      plain_unbatched: one call per product, the reference's thresholds;
      plain: one batched call, the same thresholds;
      learned: one batched call, the trained cost model choosing per product;
    each the mean of `reps` runs after a warm-up, L2 flushed before each.
    e2e: the learned batch through the host API (operands copied in, products
    copied out).  Every product of the learned run is checked modulo three
    64-bit primes."""
    import numpy as np
    import torch
    import fastfib_b200 as ff
    from fastfib_b200.workload import uneven_products
    ff.init(1 << 22)
    pairs = uneven_products(seed=seed, count=count)
    dev = torch.device("cuda")
    flat_a = torch.from_numpy(np.concatenate([a for a, _ in pairs]).view(np.int64)).to(dev)
    flat_b = torch.from_numpy(np.concatenate([b for _, b in pairs]).view(np.int64)).to(dev)
    out_len = sum(a.size + b.size + 1 for a, b in pairs)
    out = torch.empty(out_len, dtype=torch.int64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    jobs, oa, ob, oo, offs = [], 0, 0, 0, []
    for a, b in pairs:
        jobs.append({"a": flat_a.data_ptr() + 8 * oa, "b": flat_b.data_ptr() + 8 * ob, "na": a.size, "nb": b.size,
                     "bits_a": 64 * a.size, "bits_b": 64 * b.size, "out": out.data_ptr() + 8 * oo})
        offs.append(oo)
        oa, ob, oo = oa + a.size, ob + b.size, oo + a.size + b.size + 1

    # a stream of our own, given to the library and timed with events
    # recorded on it (the library runs each call on the stream it is given)
    ts_stream = torch.cuda.Stream()

    def timed(fn):
        ts = []
        for r in range(reps + 1):
            flush.fill_(r & 0xFF)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(ts_stream)
            fn()
            e1.record(ts_stream)
            torch.cuda.synchronize()
            if r:
                ts.append(e0.elapsed_time(e1))
        return statistics.mean(ts)

    stream = ts_stream.cuda_stream
    res = {}
    for m in ("plain", "learned"):
        js = ff.device_jobs([dict(j, method=m) for j in jobs])  # job records built once, outside the clock
        res[m] = timed(lambda: ff.mul_batch_device(js, stream))
    js = ff.device_jobs([dict(j, method="plain") for j in jobs])
    res["plain_unbatched"] = timed(lambda: [ff.mul_batch_device(js[i:i + 1], stream) for i in range(len(js))])
    # correctness of the learned run (the last one executed above was plain
    # unbatched; run learned once more and check every product)
    ff.mul_batch_device([dict(j, method="learned") for j in jobs], stream)
    torch.cuda.synchronize()
    got = out.cpu().numpy().view(np.uint64)
    with open(GOLD_FP) as f:
        primes = [int(p) for p in json.load(f)["primes"]][:3]
    ok = True
    for (a, b), o in zip(pairs, offs):
        x, y = int.from_bytes(a.tobytes(), "little"), int.from_bytes(b.tobytes(), "little")
        z = int.from_bytes(got[o:o + a.size + b.size + 1].tobytes(), "little")
        if any(z % p != (x % p) * (y % p) % p for p in primes) or z.bit_length() > 64 * (a.size + b.size):
            ok = False
            break
    # end to end through the host API (pinned staging inside the library,
    # sized by a first full call)
    ff.mul_batch(pairs, "learned")
    t = time.perf_counter()
    ff.mul_batch(pairs, "learned")
    e2e = (time.perf_counter() - t) * 1e3
    in_bytes = 8 * (int(flat_a.numel()) + int(flat_b.numel()))
    # the floor of that host call: the same bytes over PCIe each way, pinned
    # host buffers, one copy each (timed with events on a stream of our own)
    hin = torch.empty(in_bytes, dtype=torch.uint8, pin_memory=True)
    hout = torch.empty(8 * out_len, dtype=torch.uint8, pin_memory=True)
    dbuf = torch.empty(max(in_bytes, 8 * out_len), dtype=torch.uint8, device=dev)
    with torch.cuda.stream(ts_stream):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(ts_stream)
        dbuf[:in_bytes].copy_(hin, non_blocking=True)
        e1.record(ts_stream)
        hout.copy_(dbuf[:8 * out_len], non_blocking=True)
        e2.record(ts_stream)
    torch.cuda.synchronize()
    pcie = {"h2d_ms": e0.elapsed_time(e1), "d2h_ms": e1.elapsed_time(e2)}
    del hin, hout, dbuf
    # where the plain batch's device time goes: every launch bracketed by
    # events, per kernel family (one extra call, outside the timed runs)
    ff.profile(True)
    ff.mul_batch_device([dict(j, method="plain") for j in jobs], stream)
    torch.cuda.synchronize()
    fam = {k: {"launches": v["launches"], "ms": v["ms"]} for k, v in ff.profile_read().items() if v["launches"]}
    ff.profile(False)
    # device-only times: the batch's launches captured once and replayed
    # (host planning outside the clock)
    graph_ms = {m: ff.time_batch([dict(j, method=m) for j in jobs], reps=3) for m in ("plain", "learned")}
    cpu = None
    from oracle import Reference, reference_available
    if reference_available():
        ref = Reference()
        cpu = {"value": ref.time_mul_batch(pairs) * 1e3, "unit": "ms", "cores": ref.cpus(), "kind": "reference",
               "sample": f"the same {count} products by the reference's big_mul, one after another (each on "
                         f"all pool threads), NTT tables built first; one run"}
    return {"workload": f"{count} products, operands log-uniform 2^10..2^24 bits, aspect <= 16, seed {seed}",
            "cpu_baseline": cpu,
            "plain_unbatched_ms": res["plain_unbatched"], "plain_ms": res["plain"], "learned_ms": res["learned"],
            "learned_vs_plain": res["plain"] / res["learned"],
            "batched_learned_vs_plain_unbatched": res["plain_unbatched"] / res["learned"],
            "e2e_ms": e2e, "h2d_bytes": in_bytes, "d2h_bytes": 8 * out_len, "pcie_copies_ms": pcie,
            "graph_replay_device_ms": graph_ms, "plain_families": fam,
            "timing": "plain / learned / unbatched: CUDA events on the call's stream around the whole call "
                      "(host planning included); graph_replay_device_ms: the launches alone; e2e_ms: the "
                      "host API with operands and products in host memory",
            "bit_exact": ok,
            "l2": "flushed before every timed run"}


def run_uneven_sharded(world, rank, count=4096, seed=4, reps=3):
    """The uneven product stream split over the ranks by predicted cost
    (fastfib_b200/shard.py: longest-processing-time over the library's own
    plans), each rank's share one batched call on its GPU (operands resident),
    timed with CUDA events on the call's stream, the max over ranks; then the
    products gathered on rank 0 over the process group and checked there
    modulo three 64-bit primes.  Every rank takes the same collective steps."""
    import numpy as np
    import torch
    import torch.distributed as dist
    import fastfib_b200 as ff
    from fastfib_b200.shard import gather_products, imbalance, partition, product_cost
    from fastfib_b200.workload import uneven_products
    ff.init(1 << 22)
    pairs = uneven_products(seed=seed, count=count)
    costs = [product_cost(a.size, b.size, False) for a, b in pairs]
    shares = partition(costs, world)
    share = shares[rank]
    dev = torch.device("cuda")
    mine = [pairs[i] for i in share]
    fa = torch.from_numpy(np.concatenate([a for a, _ in mine]).view(np.int64)).to(dev)
    fb = torch.from_numpy(np.concatenate([b for _, b in mine]).view(np.int64)).to(dev)
    out = torch.empty(sum(a.size + b.size + 1 for a, b in mine), dtype=torch.int64, device=dev)
    jobs, oa, ob, oo, offs = [], 0, 0, 0, []
    for a, b in mine:
        jobs.append({"a": fa.data_ptr() + 8 * oa, "b": fb.data_ptr() + 8 * ob, "na": a.size, "nb": b.size,
                     "bits_a": 64 * a.size, "bits_b": 64 * b.size, "out": out.data_ptr() + 8 * oo, "method": "plain"})
        offs.append(oo)
        oa, ob, oo = oa + a.size, ob + b.size, oo + a.size + b.size + 1
    ts_stream = torch.cuda.Stream()
    ff.mul_batch_device(jobs, ts_stream.cuda_stream)
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ts_stream)
        ff.mul_batch_device(jobs, ts_stream.cuda_stream)
        e1.record(ts_stream)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    t = torch.tensor([statistics.mean(ts)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    host = out.cpu().numpy().view(np.uint64)
    local = {i: host[o: o + a.size + b.size + 1] for i, o, (a, b) in zip(share, offs, mine)}
    dist.barrier()
    t0 = time.perf_counter()
    got = gather_products(local, count, dst=0)
    gather_ms = (time.perf_counter() - t0) * 1e3
    if rank != 0:
        return None
    with open(GOLD_FP) as f:
        primes = [int(p) for p in json.load(f)["primes"]][:3]
    ok = all(got[i] is not None for i in range(count))
    for (a, b), z in zip(pairs, got):
        if not ok:
            break
        x, y = int.from_bytes(a.tobytes(), "little"), int.from_bytes(b.tobytes(), "little")
        zz = int.from_bytes(z.tobytes(), "little")
        ok = all(zz % p == (x % p) * (y % p) % p for p in primes)
    return {"workload": f"{count} products, operands log-uniform 2^10..2^24 bits, aspect <= 16, seed {seed}, "
                        f"split by product over {world} ranks (plain dispatch)",
            "ms": float(t.item()), "ranks": world, "products_per_rank": [len(x) for x in shares],
            "cost_imbalance": imbalance(costs, shares), "gather_ms": gather_ms, "bit_exact": ok,
            "scaling": "strong (one fixed batch)",
            "timing": "CUDA events around each rank's batched call on its stream, max over ranks"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--n", type=int, default=10**8)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-f1e9", action="store_true", help="skip the extra F(10^9) measurement")
    ap.add_argument("--config", default="fib", choices=["fib", "ntt", "ntt-suite", "uneven", "decimal"],
                    help="fib: F(n) (the headline); ntt: one NTT product of --limbs limbs; "
                         "uneven: the uneven product stream, plain against learned dispatch")
    ap.add_argument("--no-uneven", action="store_true", help="skip the uneven-stream figures in the fib line")
    ap.add_argument("--no-decimal", action="store_true", help="skip the decimal-conversion figures in the fib line")
    ap.add_argument("--no-ntt", action="store_true", help="skip the L = 2^24 NTT-pass roofline in the fib line")
    ap.add_argument("--limbs", type=int, default=1 << 22)
    ap.add_argument("--square", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.config == "ntt":
        return run_ntt_microbench(args)
    if args.config == "ntt-suite":
        r = ntt_suite(steps=args.steps, warmup=args.warmup, cpu=not args.no_cpu_baseline)
        print(json.dumps({"metric": "NTT multiply ms (microbench: 2^14..2^22 limbs, squares and products, "
                                    "plan / forced 2^k / forced 3 2^k)", "unit": "ms", "higher_is_better": False,
                          "steps": args.steps, "warmup": args.warmup, "dtype": "u32", "config": r}), flush=True)
        return 0 if r["bit_exact"] else 1
    if args.config == "decimal":
        import fastfib_b200 as ff
        ff.set_device(0)
        r = run_decimal(args.n, reps=args.steps)
        print(json.dumps({"metric": "decimal conversion of F(n) ms (device)", "value": r["device_ms"], "unit": "ms",
                          "higher_is_better": False, "steps": args.steps, "dtype": "u32", "config": r}), flush=True)
        return 0 if r["bit_exact"] else 1
    if args.config == "uneven":
        r = run_uneven(reps=args.steps)
        print(json.dumps({"metric": "uneven product stream ms (4096 products), learned vs plain dispatch",
                          "value": r["learned_ms"], "unit": "ms", "higher_is_better": False, "steps": args.steps,
                          "dtype": "u32", "config": r}), flush=True)
        return 0 if r["bit_exact"] else 1

    import torch
    import torch.distributed as dist
    import fastfib_b200 as ff
    from datetime import timedelta

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    ff.set_device(local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def barrier():
        if world > 1:
            dist.barrier()

    # warm-up: tables, arena and every kernel loaded; then which kernel family
    # dominates (a profiled run after the warm one), then the chain's CUDA
    # graph (captured on its second run with the timed profiling mask)
    r = ff.fibonacci(args.n)
    ff.profile(True)
    ff.fibonacci(args.n)
    prof = ff.profile_read()
    dominant = max(prof, key=lambda k: prof[k]["ms"])
    ok = fingerprint_ok(args.n, r)
    if ok is False:
        raise SystemExit(f"F({args.n}) does not match its golden fingerprint")
    ff.profile(False)
    for i in range(max(args.warmup - 1, 2)):
        r = ff.fibonacci(args.n)
    dev_ms, e2e_ms = [], []
    launches0 = ff.launch_count()
    torch.cuda.synchronize()
    barrier()
    with ClockSampler(local) as clk:
        t_load = time.perf_counter()
        for i in range(args.steps):
            flush.fill_(i & 0xFF)
            torch.cuda.synchronize()
            t = time.perf_counter()
            r = ff.fibonacci(args.n)
            e2e_ms.append((time.perf_counter() - t) * 1e3)
            dev_ms.append(ff.last_chain_ms())
        torch.cuda.synchronize()
        barrier()
        launches = ff.launch_count() - launches0
        # the timed steps last milliseconds, less than nvidia-smi's sampling
        # period: the same chain keeps the GPU under load (untimed) until the
        # sampler has seen it for over a second
        while time.perf_counter() - t_load < 1.2:
            ff.fibonacci(args.n)
        torch.cuda.synchronize()
    h2d, d2h = ff.last_chain_io()
    # the roofline pass: the same K steps again with CUDA events around every
    # launch of the dominant family (events perturb the chain, so `value`
    # comes from the pass above, which has none)
    ff.profile([dominant])
    for i in range(2):
        ff.fibonacci(args.n)
    ff.profile([dominant])  # reset the totals: only these K steps count
    for i in range(args.steps):
        flush.fill_(i & 0xFF)
        torch.cuda.synchronize()
        ff.fibonacci(args.n)
    prof = ff.profile_read()[dominant]
    ff.profile(False)

    value, e2e = job_ms([sum(dev_ms), sum(e2e_ms)], args.steps, world)
    sharded = run_uneven_sharded(world, rank) if world > 1 and not args.no_uneven else None

    extra = {}
    if rank == 0 and args.n == 10**8 and world == 1 and not args.no_f1e9:
        def big(n, device_fp=False, reps=3):
            # two warm-ups (the second captures the chain's CUDA graph), then
            # the median of `reps` calls, each after an L2 flush
            for _ in range(2):
                ff.fibonacci(n)
            dev_t, e2e_t, ok_n = [], [], None
            for i in range(reps):
                flush.fill_(1)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                r = ff.fibonacci(n)
                e2e_t.append((time.perf_counter() - t0) * 1e3)
                dev_t.append(ff.last_chain_ms())
                if i == 0:
                    ok_n = fingerprint_ok(n, r, ff.fingerprint if device_fp else None)
                del r  # its pinned buffer goes back to the pool for the next call
            return {"n": n, "device_ms": statistics.median(dev_t), "e2e_ms": statistics.median(e2e_t),
                    "runs": reps, "bit_exact": ok_n}
        extra = big(10**9)
        # the split multiply: forced at F(10^9) by a 2^23 cap (the reference's
        # -DNTT_MAX_LG=23), natural at F(2*10^9)
        ff.set_max_lg(23)
        try:
            extra["cap23_split"] = big(10**9)
        finally:
            ff.set_max_lg(25)
        extra["f2e9_split"] = big(2 * 10**9)
        # F(10^10): 6.9e9 bits, checked by the device fingerprint (868 MB)
        extra["f1e10_split"] = big(10**10, device_fp=True)

    if rank == 0:
        peak, peak_src = hbm_peak()
        achieved = prof["bytes"] / (prof["ms"] * 1e-3) / 1e9 if prof["ms"] > 0 else 0.0
        traffic, compute = None, None
        if os.path.exists(TRAFFIC):
            with open(TRAFFIC) as f:
                tr = json.load(f)
            fam = tr.get(dominant, {})
            traffic = fam.get("dram_bytes_per_launch")
            if "issue_active_pct" in fam:
                # what binds the kernel: the integer pipes' issue, from the same
                # ncu capture as the traffic (committed under profiles/)
                compute = {k: fam[k] for k in ("issue_active_pct", "alu_pipe_pct", "fma_pipe_pct",
                                               "warps_active_pct") if k in fam}
                compute["source"] = tr.get("source")
        line = {
            "metric": METRIC, "value": value, "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": value, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": value / PUBLISHED_F1E8_MS if args.n == 10**8 else None, "dtype": "u32",
            "data": "synthetic (F(n) needs no input data)", "config": workload(args.n),
            "bit_exact": ok,
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_src,
                         "traffic": traffic, "launches": prof["launches"],
                         "algorithmic_bytes_per_launch": prof["bytes"] / max(1, prof["launches"]),
                         "ms_per_launch": prof["ms"] / max(1, prof["launches"]),
                         "compute": compute,
                         "note": "exact modular integer transforms: instruction issue on the integer ALU and "
                                 "FMA pipes binds them, not HBM (compute: ncu fractions of peak for this "
                                 "kernel family in the F(10^8) chain); the arithmetic alone caps the NTT "
                                 "passes at about 52 % of HBM (profiles/ntt_l2e24.md); at F(10^8) the middle "
                                 "steps are short launches bound by latency"},
            "e2e": {"value": e2e, "unit": "ms", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "f1e9": extra or None,
        }
        if sharded:
            line["uneven_sharded"] = sharded
        if not args.no_uneven and world == 1:
            line["uneven"] = run_uneven(reps=3)
        if not args.no_decimal and world == 1 and args.n == 10**8:
            line["decimal"] = run_decimal(args.n)
        if not args.no_ntt and world == 1:
            nb = ntt_microbench(1 << 22, True, 3, 3)
            line["ntt_l2e24"] = {"workload": nb["config"]["workload"], "L": nb["config"]["plan"]["L"],
                                 "ms": nb["value"], "passes": nb["ntt_passes"], "families": nb["families"],
                                 "bit_exact": nb["bit_exact"]}
        if not args.no_ntt and world == 1:
            line["ntt_suite"] = ntt_suite(cpu=not args.no_cpu_baseline)
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline(args.n)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
