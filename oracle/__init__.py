"""Test infrastructure: ctypes loaders for the two CPU checkers.

* ``Oracle``    -- our own scalar C restatement of the reference's multiply hot
                   path (oracle/fastfib_oracle.c, built by ``make -C oracle``).
* ``Reference`` -- the unmodified reference compiled from its sources with a
                   Linux shim (oracle/ref_harness.c, ``make -C oracle ref``).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, and only as the checker.  Numbers cross the boundary as numpy
uint64 limb arrays (little-endian 64-bit limbs, as the reference's Big).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_libc = ctypes.CDLL(None)
_libc.strlen.restype = ctypes.c_size_t
_libc.strlen.argtypes = [ctypes.c_void_p]
_decode_ascii = ctypes.pythonapi.PyUnicode_DecodeASCII
_decode_ascii.restype = ctypes.py_object
_decode_ascii.argtypes = [ctypes.c_void_p, ctypes.c_ssize_t, ctypes.c_char_p]

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libfastfib_ref.so")
# the reference's source tree (read only); FASTFIB_REF overrides the default
REF_SRC = os.environ.get("FASTFIB_REF", "/root/reference")

_u64p = ctypes.POINTER(ctypes.c_uint64)
_szp = ctypes.POINTER(ctypes.c_size_t)


def build(with_reference: bool = True) -> None:
    """Builds the oracle library, and the reference too when its sources exist."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if with_reference and os.path.isdir(REF_SRC):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REF_SRC}"], check=True)
        # the reference's harnesses against the library (needs the library built first)
        if os.path.exists(os.path.join(os.path.dirname(HERE), "fastfib_b200", "libfastfib_b200.so")):
            subprocess.run(["make", "-s", "-C", HERE, "dropin", f"REF={REF_SRC}"], check=True)


def int_to_limbs(x: int) -> np.ndarray:
    """Python int -> uint64 limbs, little-endian, normalized (zero is [0])."""
    if x < 0:
        raise ValueError("negative")
    n = max(1, (x.bit_length() + 63) // 64)
    return np.frombuffer(x.to_bytes(8 * n, "little"), dtype=np.uint64).copy()


def limbs_to_int(a: np.ndarray) -> int:
    return int.from_bytes(np.ascontiguousarray(a, dtype=np.uint64).tobytes(), "little")


def _arr(a: np.ndarray):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return a, a.ctypes.data_as(_u64p), a.size


class _Lib:
    prefix = ""

    def __init__(self, path: str):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -C oracle{' ref' if 'ref' in path else ''})")
        self.lib = ctypes.CDLL(path)
        p = self.prefix
        for name in ("mul", "mul_ntt"):
            f = getattr(self.lib, f"{p}{name}")
            f.restype = ctypes.c_void_p
            f.argtypes = [_u64p, ctypes.c_size_t, _u64p, ctypes.c_size_t, ctypes.c_int, _szp]
        f = getattr(self.lib, f"{p}fibonacci")
        f.restype = ctypes.c_void_p
        f.argtypes = [ctypes.c_uint64, _szp]
        f = getattr(self.lib, f"{p}to_string")
        f.restype = ctypes.c_void_p
        f.argtypes = [_u64p, ctypes.c_size_t]
        getattr(self.lib, f"{p}free").argtypes = [ctypes.c_void_p]
        getattr(self.lib, f"{p}ntt_init").argtypes = [ctypes.c_size_t]
        getattr(self.lib, f"{p}ntt_max_L").restype = ctypes.c_size_t
        getattr(self.lib, f"{p}set_ntt_max_L").argtypes = [ctypes.c_size_t]

    def _take(self, ptr, n) -> np.ndarray:
        out = np.ctypeslib.as_array(ctypes.cast(ptr, _u64p), shape=(n,)).copy()
        getattr(self.lib, f"{self.prefix}free")(ptr)
        return out

    def _mul(self, name, a, b, square):
        a, pa, na = _arr(a)
        if square:
            b, pb, nb = a, pa, na
        else:
            b, pb, nb = _arr(b)
        n = ctypes.c_size_t()
        ptr = getattr(self.lib, f"{self.prefix}{name}")(pa, na, pb, nb, int(square), ctypes.byref(n))
        return self._take(ptr, n.value)

    def mul(self, a, b=None, square=False):
        """big_mul / big_sqr: the threshold dispatch."""
        return self._mul("mul", a, a if b is None else b, square or b is None)

    def mul_ntt(self, a, b=None, square=False):
        """big_mul_ntt: the NTT multiply (square when b is None)."""
        return self._mul("mul_ntt", a, a if b is None else b, square or b is None)

    def fibonacci(self, n: int) -> np.ndarray:
        k = ctypes.c_size_t()
        ptr = getattr(self.lib, f"{self.prefix}fibonacci")(n, ctypes.byref(k))
        return self._take(ptr, k.value)

    def to_string(self, a) -> str:
        a, pa, na = _arr(a)
        ptr = getattr(self.lib, f"{self.prefix}to_string")(pa, na)
        # one pass from the C string to a str, as fastfib_b200.to_decimal does
        s = _decode_ascii(ptr, _libc.strlen(ptr), None)
        getattr(self.lib, f"{self.prefix}free")(ptr)
        return s

    def ntt_init(self, max_limbs: int) -> None:
        getattr(self.lib, f"{self.prefix}ntt_init")(max_limbs)

    def ntt_max_L(self) -> int:
        return getattr(self.lib, f"{self.prefix}ntt_max_L")()

    def set_ntt_max_L(self, L: int) -> None:
        getattr(self.lib, f"{self.prefix}set_ntt_max_L")(L)


class FoPlan(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("lg", ctypes.c_uint32), ("r3", ctypes.c_uint32),
                ("split", ctypes.c_uint32), ("L", ctypes.c_uint64), ("conv", ctypes.c_uint64),
                ("ca", ctypes.c_uint64), ("cb", ctypes.c_uint64), ("ka", ctypes.c_uint64),
                ("kb", ctypes.c_uint64), ("Lbig", ctypes.c_uint64)]


class Oracle(_Lib):
    """Our scalar C restatement (oracle/fastfib_oracle.c)."""
    prefix = "fo_"

    def __init__(self, path: str = ORACLE_SO):
        super().__init__(path)
        self.lib.fo_ntt_plan.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(FoPlan)]
        self.lib.fo_ntt_plan.restype = ctypes.c_int
        self.lib.fo_set_max_lg.argtypes = [ctypes.c_int]
        self.lib.fo_fingerprint.argtypes = [_u64p, ctypes.c_size_t, _u64p]
        self.lib.fo_mul_ntt_forced.restype = ctypes.c_void_p
        self.lib.fo_mul_ntt_forced.argtypes = [_u64p, ctypes.c_size_t, _u64p, ctypes.c_size_t, ctypes.c_int,
                                               ctypes.c_uint32, ctypes.c_uint64, _szp]

    def mlp_nparam(self) -> int:
        self.lib.fo_mlp_nparam.restype = ctypes.c_size_t
        return self.lib.fo_mlp_nparam()

    def mlp_predict(self, params: np.ndarray, X: np.ndarray) -> np.ndarray:
        """Every output of the cost model for the rows of X (float32, n x 8)."""
        params = np.ascontiguousarray(params, dtype=np.float32)
        X = np.ascontiguousarray(X, dtype=np.float32)
        out = np.zeros((X.shape[0], 4), dtype=np.float64)
        fp = ctypes.POINTER(ctypes.c_float)
        self.lib.fo_mlp_predict.argtypes = [fp, fp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_double)]
        self.lib.fo_mlp_predict(params.ctypes.data_as(fp), X.ctypes.data_as(fp), X.shape[0],
                                out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out

    def mlp_grad(self, params: np.ndarray, X: np.ndarray, method: np.ndarray, y: np.ndarray):
        """(loss, gradient) of the cost model in double precision."""
        params = np.ascontiguousarray(params, dtype=np.float32)
        X = np.ascontiguousarray(X, dtype=np.float32)
        method = np.ascontiguousarray(method, dtype=np.int32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        grad = np.zeros(self.mlp_nparam(), dtype=np.float64)
        fp = ctypes.POINTER(ctypes.c_float)
        self.lib.fo_mlp_grad.argtypes = [fp, fp, ctypes.POINTER(ctypes.c_int32), fp, ctypes.c_size_t,
                                         ctypes.POINTER(ctypes.c_double)]
        self.lib.fo_mlp_grad.restype = ctypes.c_double
        loss = self.lib.fo_mlp_grad(params.ctypes.data_as(fp), X.ctypes.data_as(fp),
                                    method.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), y.ctypes.data_as(fp),
                                    X.shape[0], grad.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return loss, grad

    def set_max_lg(self, lg: int) -> None:
        self.lib.fo_set_max_lg(lg)

    def plan(self, bits_a: int, bits_b: int, square: bool = False) -> FoPlan:
        p = FoPlan()
        self.lib.fo_ntt_plan(bits_a, bits_b, int(square), ctypes.byref(p))
        return p

    def mul_ntt_forced(self, a, b, width: int, L: int, square=False):
        a, pa, na = _arr(a)
        b, pb, nb = (a, pa, na) if square else _arr(b)
        n = ctypes.c_size_t()
        ptr = self.lib.fo_mul_ntt_forced(pa, na, pb, nb, int(square), width, L, ctypes.byref(n))
        return self._take(ptr, n.value)

    def residues(self, a, b, width: int, L: int, k: int, square=False) -> np.ndarray:
        """Prime k's scaled convolution of a * b at (width, L): L uint32 words."""
        a, pa, na = _arr(a)
        b, pb, nb = (a, pa, na) if square else _arr(b)
        y = np.zeros(L, dtype=np.uint32)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        self.lib.fo_residues.argtypes = [_u64p, ctypes.c_size_t, _u64p, ctypes.c_size_t, ctypes.c_int,
                                         ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, u32p]
        if self.lib.fo_residues(pa, na, pb, nb, int(square), width, L, k, y.ctypes.data_as(u32p)):
            raise ValueError(f"residues: L={L} too short, or prime {k} / width {width} out of range")
        return y

    def crt_residues(self, y: np.ndarray, L: int, conv: int, width: int, limbs: int) -> np.ndarray:
        """The product from all three primes' residues (y: 3 x L uint32)."""
        y = np.ascontiguousarray(y, dtype=np.uint32).reshape(-1)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        self.lib.fo_crt_residues.restype = ctypes.c_void_p
        self.lib.fo_crt_residues.argtypes = [u32p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32,
                                             ctypes.c_size_t, _szp]
        n = ctypes.c_size_t()
        ptr = self.lib.fo_crt_residues(y.ctypes.data_as(u32p), L, conv, width, limbs, ctypes.byref(n))
        return self._take(ptr, n.value)

    def fingerprint(self, a) -> tuple:
        a, pa, na = _arr(a)
        out = (ctypes.c_uint64 * 6)()
        self.lib.fo_fingerprint(pa, na, out)
        return tuple(int(v) for v in out)


class Reference(_Lib):
    """The unmodified reference built from its sources (oracle/_ref)."""
    prefix = "ffref_"

    def __init__(self, path: str = REF_SO):
        super().__init__(path)
        self.lib.ffref_seconds.restype = ctypes.c_double
        self.lib.ffref_cpus.restype = ctypes.c_int

    def seconds(self) -> float:
        return self.lib.ffref_seconds()

    def cpus(self) -> int:
        return self.lib.ffref_cpus()

    def time_mul(self, a, b=None, square=False, reps=3) -> float:
        """Seconds of the fastest of `reps` big_mul / big_sqr calls, timed in C."""
        a, pa, na = _arr(a)
        if square or b is None:
            pb, nb = pa, na
        else:
            b, pb, nb = _arr(b)
        f = self.lib.ffref_time_mul
        f.restype = ctypes.c_double
        f.argtypes = [_u64p, ctypes.c_size_t, _u64p, ctypes.c_size_t, ctypes.c_int, ctypes.c_int]
        return f(pa, na, pb, nb, int(bool(square or b is None)), reps)

    def time_mul_batch(self, pairs) -> float:
        """Seconds for big_mul over every (a, b) pair, one after another, timed in C."""
        na = np.array([a.size for a, _ in pairs], dtype=np.uint64)
        nb = np.array([b.size for _, b in pairs], dtype=np.uint64)
        aoff = np.concatenate([[0], np.cumsum(na)[:-1]]).astype(np.uint64)
        boff = np.concatenate([[0], np.cumsum(nb)[:-1]]).astype(np.uint64)
        A = np.ascontiguousarray(np.concatenate([a for a, _ in pairs]), dtype=np.uint64)
        B = np.ascontiguousarray(np.concatenate([b for _, b in pairs]), dtype=np.uint64)
        f = self.lib.ffref_time_mul_batch
        f.restype = ctypes.c_double
        f.argtypes = [_u64p, _szp, _szp, _u64p, _szp, _szp, ctypes.c_size_t]
        sp = lambda x: x.ctypes.data_as(_szp)  # noqa: E731
        return f(A.ctypes.data_as(_u64p), sp(aoff), sp(na), B.ctypes.data_as(_u64p), sp(boff), sp(nb), len(pairs))


def reference_available() -> bool:
    return os.path.exists(REF_SO)
