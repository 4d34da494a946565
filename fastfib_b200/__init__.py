"""fastfib_b200: the reference's multiply hot path on a B200.

A ctypes mirror of the two C interfaces of ``libfastfib_b200.so``:

* the reference's own surface (include/fastfib.h): ``big_mul``, ``big_sqr``,
  ``big_mul_ntt``, ``fibonacci``, ``big_to_string``, ``ntt_init`` and the
  transform cap ``g_ntt_max_L``, with the same names and meaning;
* the thin GPU ABI (include/ffg.h): plans, device-pointer products, the
  device fast-doubling chain.

Numbers cross as numpy uint64 limb arrays (little-endian 64-bit limbs, the
reference's Big).  There is no CPU fallback: if the library or a GPU is
missing, calls raise.
"""
from __future__ import annotations

import ctypes
import os
import weakref

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libfastfib_b200.so")
TUNING_PATH = os.path.join(PKG, "tuning.txt")  # written by python -m fastfib_b200.tune

_u64p = ctypes.POINTER(ctypes.c_uint64)
_szp = ctypes.POINTER(ctypes.c_size_t)


class Big(ctypes.Structure):
    """The reference's Big (src/common.h:29-33)."""
    _fields_ = [("d", _u64p), ("n", ctypes.c_size_t)]


class Plan(ctypes.Structure):
    """ffg_plan (include/ffg.h)."""
    _fields_ = [("width", ctypes.c_uint32), ("lg", ctypes.c_uint32), ("r3", ctypes.c_uint32),
                ("split", ctypes.c_uint32), ("L", ctypes.c_uint64), ("conv", ctypes.c_uint64),
                ("ca", ctypes.c_uint64), ("cb", ctypes.c_uint64), ("ka", ctypes.c_uint64),
                ("kb", ctypes.c_uint64), ("Lbig", ctypes.c_uint64), ("kernel", ctypes.c_uint32),
                ("row_lg", ctypes.c_uint32)]

    def as_dict(self) -> dict:
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class Job(ctypes.Structure):
    """ffg_job (include/ffg.h)."""
    _fields_ = [("a", _u64p), ("b", _u64p), ("na", ctypes.c_uint64), ("nb", ctypes.c_uint64),
                ("bits_a", ctypes.c_uint64), ("bits_b", ctypes.c_uint64), ("out", _u64p),
                ("nout", ctypes.c_uint64), ("square", ctypes.c_int32), ("method", ctypes.c_int32)]


# methods of a batched product (FFG_M_*)
METHODS = {"plain": -1, "school": 0, "ntt": 1, "ntt_pow2": 2, "ntt_r3": 3, "learned": 4}
# cost-model outputs, in order (FFG_M_SCHOOL .. FFG_M_NTT_R3)
MODEL_METHODS = ("school", "ntt", "ntt_pow2", "ntt_r3")
MLP_D, MLP_H, MLP_K = 8, 32, 4
MLP_NPARAM = MLP_H * MLP_D + MLP_H + MLP_H * MLP_H + MLP_H + MLP_K * MLP_H + MLP_K


class FfgError(RuntimeError):
    pass


_lib = None


def lib() -> ctypes.CDLL:
    """Loads libfastfib_b200.so (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FfgError(f"{LIB_PATH} is not built: run python -m fastfib_b200.build")
    L = ctypes.CDLL(LIB_PATH)
    L.ffg_init.argtypes = [ctypes.c_size_t]
    L.ffg_ntt_max_L.restype = ctypes.c_size_t
    L.ffg_set_ntt_max_L.argtypes = [ctypes.c_size_t]
    L.ffg_plan_select.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(Plan)]
    L.ffg_mul_host.argtypes = [_u64p, _szp, _u64p, ctypes.c_size_t, _u64p, ctypes.c_size_t, ctypes.c_int]
    L.ffg_mul_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64,
                                 ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_int,
                                 ctypes.c_void_p]
    L.ffg_mul_residues.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64,
                                   ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_int,
                                   ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p]
    L.ffg_crt_residues.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64,
                                   ctypes.c_size_t, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p]
    L.ffg_fib_chain.argtypes = [ctypes.c_uint64, ctypes.c_int, _u64p, ctypes.c_size_t, _u64p,
                                ctypes.c_size_t, ctypes.POINTER(_u64p), _szp]
    L.ffg_last_chain_ms.restype = ctypes.c_double
    L.ffg_profile.argtypes = [ctypes.c_uint32]
    L.ffg_last_chain_io.argtypes = [ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
    L.ffg_set_device.argtypes = [ctypes.c_int]
    L.ffg_set_max_lg.argtypes = [ctypes.c_int]
    L.ff_set_max_lg.argtypes = [ctypes.c_int]
    L.ffg_profile_read.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double)]
    L.ffg_launch_count.restype = ctypes.c_uint64
    L.ffg_last_error.restype = ctypes.c_char_p
    L.ffg_free.argtypes = [ctypes.c_void_p]
    L.ffg_mul_batch_host.argtypes = [ctypes.POINTER(Job), ctypes.c_size_t]
    _fp = ctypes.POINTER(ctypes.c_float)
    _ip = ctypes.POINTER(ctypes.c_int32)
    L.ffg_mlp_features.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, _fp]
    L.ffg_mlp_train.argtypes = [_fp, _fp, _ip, _fp, ctypes.c_size_t, ctypes.c_int, ctypes.c_float, _fp]
    L.ffg_mlp_grad.argtypes = [_fp, _fp, _ip, _fp, ctypes.c_size_t, _fp, _fp]
    L.ffg_mlp_predict.argtypes = [_fp, _fp, ctypes.c_size_t, _fp]
    L.ffg_mlp_set.argtypes = [_fp]
    L.ffg_time_batch.argtypes = [ctypes.POINTER(Job), ctypes.c_size_t, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.ffg_set_geometry.argtypes = [ctypes.c_uint32] * 4
    L.ffg_get_geometry.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32),
                                   ctypes.POINTER(ctypes.c_uint32)]
    L.ffg_load_tuning.argtypes = [ctypes.c_char_p]
    L.ffg_last_decimal_ms.restype = ctypes.c_double
    L.ffg_to_decimal_host.argtypes = [_u64p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p), _szp,
                                      ctypes.POINTER(ctypes.c_int)]
    L.ffg_to_decimal_device.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p), _szp,
                                        ctypes.POINTER(ctypes.c_int)]
    L.ffg_mul_batch_device.argtypes = [ctypes.POINTER(Job), ctypes.c_size_t, ctypes.c_void_p]
    L.ffg_release.argtypes = [ctypes.c_void_p]
    for name in ("big_mul", "big_mul_ntt", "big_mul_toom3"):
        getattr(L, name).restype = Big
        getattr(L, name).argtypes = [ctypes.POINTER(Big), ctypes.POINTER(Big)]
    L.big_sqr.restype = Big
    L.big_sqr.argtypes = [ctypes.POINTER(Big)]
    L.fibonacci.restype = Big
    L.fibonacci.argtypes = [ctypes.c_uint64]
    L.big_to_string.restype = ctypes.c_void_p
    L.big_to_string.argtypes = [ctypes.POINTER(Big)]
    L.big_free.argtypes = [ctypes.POINTER(Big)]
    L.ntt_init.argtypes = [ctypes.c_size_t]
    L.plat_seconds.restype = ctypes.c_double
    _lib = L
    # the autotuner's geometry table and cost model, measured on a B200
    if os.path.exists(TUNING_PATH) and not os.environ.get("FASTFIB_B200_NO_TUNING"):
        _check(L.ffg_load_tuning(TUNING_PATH.encode()))
    return L


def _check(rc: int) -> None:
    if rc:
        raise FfgError(f"ffg error {rc}: {lib().ffg_last_error().decode()}")


def _arr(a) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    if a.size == 0:
        a = np.zeros(1, dtype=np.uint64)
    return a


def _view(a: np.ndarray) -> Big:
    n = a.size
    while n > 1 and a[n - 1] == 0:
        n -= 1
    return Big(a.ctypes.data_as(_u64p), n)


def _release(big: Big) -> None:
    lib().big_free(ctypes.byref(big))


def _take(b: Big) -> np.ndarray:
    """The Big's limbs as a numpy array that owns them (no copy); the limbs
    are released with big_free when the array is collected."""
    out = np.ctypeslib.as_array(b.d, shape=(b.n,))
    weakref.finalize(out, _release, Big(b.d, b.n))
    return out


def int_to_limbs(x: int) -> np.ndarray:
    n = max(1, (x.bit_length() + 63) // 64)
    return np.frombuffer(x.to_bytes(8 * n, "little"), dtype=np.uint64).copy()


def limbs_to_int(a: np.ndarray) -> int:
    return int.from_bytes(np.ascontiguousarray(a, dtype=np.uint64).tobytes(), "little")


# ------------------------------------------------------------ the C surface

def g_ntt_max_L() -> int:
    return ctypes.c_size_t.in_dll(lib(), "g_ntt_max_L").value


def set_g_ntt_max_L(L: int) -> None:
    """Overrides the transform cap, as tests/nttfuzz.c:33-39 does."""
    ctypes.c_size_t.in_dll(lib(), "g_ntt_max_L").value = L


def ntt_init(max_limbs: int) -> None:
    lib().ntt_init(max_limbs)


def set_max_lg(lg: int) -> None:
    """The reference's NTT_MAX_LG at run time (25 by default): lower values send
    long products to the split multiply (its -DNTT_MAX_LG=23 / 12 / 10 builds)."""
    _check(lib().ff_set_max_lg(lg))


def big_mul(a, b) -> np.ndarray:
    a, b = _arr(a), _arr(b)
    A, B = _view(a), _view(b)
    return _take(lib().big_mul(ctypes.byref(A), ctypes.byref(B)))


def big_sqr(a) -> np.ndarray:
    a = _arr(a)
    A = _view(a)
    return _take(lib().big_sqr(ctypes.byref(A)))


def big_mul_ntt(a, b=None) -> np.ndarray:
    """big_mul_ntt; b None squares (the reference passes a == b)."""
    a = _arr(a)
    A = _view(a)
    if b is None:
        return _take(lib().big_mul_ntt(ctypes.byref(A), ctypes.byref(A)))
    b = _arr(b)
    B = _view(b)
    return _take(lib().big_mul_ntt(ctypes.byref(A), ctypes.byref(B)))


def fibonacci(n: int) -> np.ndarray:
    return _take(lib().fibonacci(n))


def big_to_string(a) -> str:
    a = _arr(a)
    A = _view(a)
    p = lib().big_to_string(ctypes.byref(A))
    s = ctypes.string_at(p).decode()
    ctypes.CDLL(None).free(ctypes.c_void_p(p))
    return s


def last_decimal_ms() -> float:
    return lib().ffg_last_decimal_ms()


def decimal_cache_clear() -> None:
    lib().ffg_decimal_cache_clear()


FP_PRIMES = (18446744073709551557, 18446744073709551533, 9223372036854775783, 4611686018427387847)


def fingerprint(a=None, device_ptr: int = 0, n: int = 0) -> list:
    """ffg_fingerprint_host / _device: [bits, low 64 bits, x mod each of
    FP_PRIMES], computed on the GPU."""
    out = (ctypes.c_uint64 * 6)()
    if device_ptr:
        _check(lib().ffg_fingerprint_device(ctypes.cast(device_ptr, _u64p), n, out))
    else:
        a = _arr(a)
        _check(lib().ffg_fingerprint_host(a.ctypes.data_as(_u64p), a.size, out))
    return [int(v) for v in out]


def tickets_in_use() -> int:
    """ffg_tickets_in_use: non-zero words of the carry-settle ticket pool (0 when idle)."""
    f = lib().ffg_tickets_in_use
    f.restype = ctypes.c_int64
    return f()


def to_decimal(a, device_ptr: int = 0, n: int = 0):
    """ffg_to_decimal_host (or _device with device_ptr, n limbs): (digits,
    True) from the device path, or (None, False) when it declined."""
    out, nout, done = ctypes.c_void_p(), ctypes.c_size_t(), ctypes.c_int()
    if device_ptr:
        _check(lib().ffg_to_decimal_device(device_ptr, n, ctypes.byref(out), ctypes.byref(nout), ctypes.byref(done)))
    else:
        a = _arr(a)
        _check(lib().ffg_to_decimal_host(a.ctypes.data_as(_u64p), a.size, ctypes.byref(out), ctypes.byref(nout),
                                         ctypes.byref(done)))
    if not done.value:
        return None, False
    s = _ascii_str(out.value, nout.value)
    lib().ffg_free(out)
    return s, True


_SINK = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p)


def to_decimal_stream(a):
    """ffg_to_decimal_stream: (list of digit slices as str, True) from the
    streamed device path, or ([], False) when it declined."""
    pieces = []

    def sink(ptr, n, user):
        pieces.append(_ascii_str(ptr, n))

    cb = _SINK(sink)
    a = _arr(a)
    nd, done = ctypes.c_size_t(), ctypes.c_int()
    f = lib().ffg_to_decimal_stream
    f.argtypes = [_u64p, ctypes.c_size_t, _SINK, ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t),
                  ctypes.POINTER(ctypes.c_int)]
    _check(f(a.ctypes.data_as(_u64p), a.size, cb, None, ctypes.byref(nd), ctypes.byref(done)))
    if not done.value:
        return [], False
    if sum(len(x) for x in pieces) != nd.value:
        raise FfgError("streamed digit count mismatch")
    return pieces, True


_decode_ascii = ctypes.pythonapi.PyUnicode_DecodeASCII
_decode_ascii.restype = ctypes.py_object
_decode_ascii.argtypes = [ctypes.c_void_p, ctypes.c_ssize_t, ctypes.c_char_p]


def _ascii_str(ptr: int, n: int) -> str:
    """A Python str of the n ASCII bytes at ptr, decoded in one pass (no
    intermediate bytes object)."""
    return _decode_ascii(ptr, n, None)


# ------------------------------------------------------------------ the GPU ABI

def init(max_limbs: int) -> None:
    _check(lib().ffg_init(max_limbs))


def ntt_max_L() -> int:
    """The GPU layer's transform cap (ffg_ntt_max_L)."""
    return lib().ffg_ntt_max_L()


def plan(bits_a: int, bits_b: int, square: bool = False) -> dict:
    p = Plan()
    _check(lib().ffg_plan_select(bits_a, bits_b, int(square), ctypes.byref(p)))
    return p.as_dict()


def mul(a, b=None) -> np.ndarray:
    """ffg_mul_host: the NTT product on the GPU (b None squares)."""
    a = _arr(a)
    sq = b is None
    b = a if sq else _arr(b)
    out = np.zeros(a.size + b.size + 1, dtype=np.uint64)
    n = ctypes.c_size_t()
    _check(lib().ffg_mul_host(out.ctypes.data_as(_u64p), ctypes.byref(n), a.ctypes.data_as(_u64p), a.size,
                              b.ctypes.data_as(_u64p), b.size, int(sq)))
    return out[: n.value].copy()


def mul_batch(pairs, method="ntt") -> list:
    """ffg_mul_batch_host: many independent products in one call.  pairs holds
    (a, b) with b None for a square; method names one of METHODS, or is a list
    with one name per product.  The products come back as views of one
    output area."""
    A = [_arr(a) for a, _ in pairs]
    B = [A[i] if b is None else _arr(b) for i, (_, b) in enumerate(pairs)]
    n = len(pairs)
    jobs = np.zeros(max(1, n), dtype=_JOB_DT)
    if n:
        na = np.fromiter((a.size for a in A), dtype=np.uint64, count=n)
        nb = np.fromiter((b.size for b in B), dtype=np.uint64, count=n)
        offs = np.concatenate([[0], np.cumsum(na + nb)[:-1]]).astype(np.uint64)
        area = np.empty(int((na + nb).sum()), dtype=np.uint64)
        jobs["a"][:n] = [a.ctypes.data for a in A]
        jobs["b"][:n] = [b.ctypes.data for b in B]
        jobs["na"][:n], jobs["nb"][:n] = na, nb
        jobs["out"][:n] = area.ctypes.data + 8 * offs
        jobs["square"][:n] = [int(b is None) for _, b in pairs]
        ms = method if isinstance(method, (list, tuple)) else [method] * n
        jobs["method"][:n] = [METHODS[m] for m in ms]
    ptr = ctypes.cast(jobs.ctypes.data, ctypes.POINTER(Job))
    _check(lib().ffg_mul_batch_host(ptr, n))
    if not n:
        return []
    nout = jobs["nout"]
    return [area[int(offs[i]): int(offs[i]) + int(nout[i])] for i in range(n)]


# ffg_job as a numpy record (the same 72-byte layout as Job)
_JOB_DT = np.dtype([("a", "<u8"), ("b", "<u8"), ("na", "<u8"), ("nb", "<u8"), ("bits_a", "<u8"),
                    ("bits_b", "<u8"), ("out", "<u8"), ("nout", "<u8"), ("square", "<i4"), ("method", "<i4")])


def device_jobs(jobs) -> np.ndarray:
    """The job records of mul_batch_device (a list of dicts as it takes) built
    column by column, to be reused across calls."""
    arr = np.zeros(len(jobs), dtype=_JOB_DT)
    arr["a"] = [d["a"] for d in jobs]
    arr["b"] = [d.get("b") or d["a"] for d in jobs]
    arr["na"] = [d["na"] for d in jobs]
    arr["nb"] = [d.get("nb", d["na"]) for d in jobs]
    arr["bits_a"] = [d["bits_a"] for d in jobs]
    arr["bits_b"] = [d.get("bits_b", d["bits_a"]) for d in jobs]
    arr["out"] = [d["out"] for d in jobs]
    arr["square"] = [int(d.get("square", False)) for d in jobs]
    arr["method"] = [METHODS[d.get("method", "ntt")] for d in jobs]
    return arr


def mul_batch_device(jobs, stream: int = 0) -> None:
    """ffg_mul_batch_device on a list of dicts with device pointers:
    a, b, na, nb, bits_a, bits_b, out (na + nb + 1 limbs), square, method --
    or on the records device_jobs built from such a list."""
    if isinstance(jobs, np.ndarray):
        assert jobs.dtype == _JOB_DT
        ptr = ctypes.cast(jobs.ctypes.data, ctypes.POINTER(Job))
        _check(lib().ffg_mul_batch_device(ptr, len(jobs), stream or None))
        return
    _check(lib().ffg_mul_batch_device(_device_jobs(jobs), len(jobs), stream or None))


def _device_jobs(jobs):
    arr = (Job * max(1, len(jobs)))()
    for i, d in enumerate(jobs):
        j = arr[i]
        j.a = ctypes.cast(d["a"], _u64p)
        j.b = ctypes.cast(d.get("b") or d["a"], _u64p)
        j.na, j.nb = d["na"], d.get("nb", d["na"])
        j.bits_a, j.bits_b = d["bits_a"], d.get("bits_b", d["bits_a"])
        j.out = ctypes.cast(d["out"], _u64p)
        j.square = int(d.get("square", False))
        j.method = METHODS[d.get("method", "ntt")]
    return arr


def time_batch(jobs, reps: int = 3) -> float:
    """ffg_time_batch: device milliseconds of one mul_batch_device call on
    `jobs` (dicts as mul_batch_device takes), the mean of reps runs."""
    ms = ctypes.c_double()
    _check(lib().ffg_time_batch(_device_jobs(jobs), len(jobs), reps, ctypes.byref(ms)))
    return ms.value


# ------------------------------------------------------------ the cost model

def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def mlp_features(bits_a: int, bits_b: int, square: bool = False) -> np.ndarray:
    f = np.zeros(MLP_D, dtype=np.float32)
    _check(lib().ffg_mlp_features(bits_a, bits_b, int(square), _fptr(f)))
    return f


def mlp_init(seed: int = 0) -> np.ndarray:
    """Initial parameters: uniform +-sqrt(6 / (fan_in + fan_out)) weights, zero biases."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_in, fan_out in ((MLP_D, MLP_H), (MLP_H, MLP_H), (MLP_H, MLP_K)):
        lim = np.sqrt(6.0 / (fan_in + fan_out))
        parts += [rng.uniform(-lim, lim, fan_in * fan_out), np.zeros(fan_out)]
    return _f32(np.concatenate(parts))


def mlp_train(params, X, method, y, epochs: int = 1000, lr: float = 1e-2):
    """ffg_mlp_train: (trained parameters, loss before each epoch)."""
    p = _f32(params).copy()
    X, y = _f32(X), _f32(y)
    m = np.ascontiguousarray(method, dtype=np.int32)
    hist = np.zeros(max(1, epochs), dtype=np.float32)
    _check(lib().ffg_mlp_train(_fptr(p), _fptr(X), m.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), _fptr(y),
                               len(y), epochs, lr, _fptr(hist)))
    return p, hist[:epochs]


def mlp_grad(params, X, method, y):
    """ffg_mlp_grad: (loss, gradient) from the GPU kernel."""
    p, X, y = _f32(params), _f32(X), _f32(y)
    m = np.ascontiguousarray(method, dtype=np.int32)
    g = np.zeros(MLP_NPARAM, dtype=np.float32)
    loss = ctypes.c_float()
    _check(lib().ffg_mlp_grad(_fptr(p), _fptr(X), m.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), _fptr(y),
                              len(y), _fptr(g), ctypes.byref(loss)))
    return loss.value, g


def mlp_predict(params, X) -> np.ndarray:
    """ffg_mlp_predict: every output for the rows of X (params None: the installed model)."""
    X = _f32(X)
    out = np.zeros((X.shape[0], MLP_K), dtype=np.float32)
    p = None if params is None else _f32(params)
    _check(lib().ffg_mlp_predict(None if p is None else _fptr(p), _fptr(X), X.shape[0], _fptr(out)))
    return out


def set_model(params) -> None:
    """ffg_mlp_set: installs the cost model for method "learned" (None removes it)."""
    p = None if params is None else _f32(params)
    _check(lib().ffg_mlp_set(None if p is None else _fptr(p)))


def load_tuning(path: str = TUNING_PATH) -> bool:
    """ffg_load_tuning: installs the autotuner's geometry table and cost
    model; False if the file does not exist."""
    if not os.path.exists(path):
        return False
    _check(lib().ffg_load_tuning(path.encode()))
    return True


def set_geometry(lg: int, r3: int, row_lg: int, wc: int) -> None:
    _check(lib().ffg_set_geometry(lg, r3, row_lg, wc))


def get_geometry(lg: int, r3: int) -> tuple:
    c, w = ctypes.c_uint32(), ctypes.c_uint32()
    _check(lib().ffg_get_geometry(lg, r3, ctypes.byref(c), ctypes.byref(w)))
    return c.value, w.value


def write_tuning(path: str, geometry, params, comment: str = "") -> None:
    """The tuning file ffg_load_tuning reads: geometry rows (lg, r3, row_lg,
    wc) and the cost model's parameters."""
    with open(path, "w") as f:
        f.write("# fastfib_b200 tuning: four-step geometry and cost model\n")
        for line in comment.splitlines():
            f.write(f"# {line}\n")
        for lg, r3, c, wc in geometry:
            f.write(f"geometry {lg} {r3} {c} {wc}\n")
        if params is not None:
            p = _f32(params)
            f.write(f"mlp {p.size} " + " ".join(f"{v:.9g}" for v in p) + "\n")


def mul_device(out_ptr: int, a_ptr: int, na: int, bits_a: int, b_ptr: int, nb: int, bits_b: int,
               square: bool = False, stream: int = 0) -> None:
    """ffg_mul_device on device pointers (e.g. torch tensors' data_ptr())."""
    _check(lib().ffg_mul_device(out_ptr, a_ptr, na, bits_a, b_ptr if not square else a_ptr, nb, bits_b,
                                int(square), stream or None))


def mul_residues(y_ptr: int, a_ptr: int, na: int, bits_a: int, b_ptr: int, nb: int, bits_b: int,
                 square: bool, prime0: int, nprimes: int, stream: int = 0) -> None:
    """ffg_mul_residues: the scaled convolution of a*b modulo primes
    [prime0, prime0 + nprimes) into y (3 * plan.L uint32 words, prime-major,
    device memory); one product's share on a GPU that shards it by prime."""
    _check(lib().ffg_mul_residues(y_ptr, a_ptr, na, bits_a, b_ptr if not square else a_ptr, nb, bits_b,
                                  int(square), prime0, nprimes, stream or None))


def crt_residues(out_ptr: int, y_ptr: int, na: int, bits_a: int, nb: int, bits_b: int, square: bool,
                 stream: int = 0) -> None:
    """ffg_crt_residues: the product (na + nb + 1 limbs into out) from the
    three primes' residues in y, as gathered from the GPUs that shared it."""
    _check(lib().ffg_crt_residues(out_ptr, y_ptr, na, bits_a, nb, bits_b, int(square), stream or None))


def fib_chain(n: int, i0: int, fkm1, fk) -> np.ndarray:
    fkm1, fk = _arr(fkm1), _arr(fk)
    out = _u64p()
    nout = ctypes.c_size_t()
    _check(lib().ffg_fib_chain(n, i0, fkm1.ctypes.data_as(_u64p), fkm1.size, fk.ctypes.data_as(_u64p),
                               fk.size, ctypes.byref(out), ctypes.byref(nout)))
    r = np.ctypeslib.as_array(out, shape=(nout.value,)).copy()
    lib().ffg_free(out)
    return r


def last_chain_ms() -> float:
    return lib().ffg_last_chain_ms()


KERNEL_FAMILIES = ("conv_small", "col_fwd", "row_conv", "col_inv", "crt", "carry", "lin", "school")


def profile(families=None) -> None:
    """Resets the per-family totals; brackets the named kernel families (all
    when families is True, none when falsy) with CUDA events from now on."""
    if families is True:
        mask = (1 << len(KERNEL_FAMILIES)) - 1
    elif not families:
        mask = 0
    else:
        mask = sum(1 << KERNEL_FAMILIES.index(f) for f in families)
    lib().ffg_profile(mask)


def last_chain_io() -> tuple:
    h, d = ctypes.c_uint64(), ctypes.c_uint64()
    lib().ffg_last_chain_io(ctypes.byref(h), ctypes.byref(d))
    return h.value, d.value


def set_device(device: int) -> None:
    _check(lib().ffg_set_device(device))


def profile_read() -> dict:
    out = {}
    for k, name in enumerate(KERNEL_FAMILIES):
        n, ms, by = ctypes.c_uint64(), ctypes.c_double(), ctypes.c_double()
        _check(lib().ffg_profile_read(k, ctypes.byref(n), ctypes.byref(ms), ctypes.byref(by)))
        out[name] = {"launches": n.value, "ms": ms.value, "bytes": by.value}
    return out


def launch_count() -> int:
    return lib().ffg_launch_count()
