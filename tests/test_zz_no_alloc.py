"""The allocation-free multiply (ffg_mul_device_noalloc) against the
allocating one (ffg_mul_device), through the C ABI.

Some callers cannot allocate device memory once they are running -- host
programs whose GPU memory is owned by a framework allocator or a fixed
start-up budget, paths that cannot afford a cudaMalloc.  This entry point
serves them from one fixed 8 MiB scratch array per GPU.  The tests run
calls in a row (different sizes, a square and a distinct product, the
one-CTA and the four-step kernels) and require bit-identical limbs, check
that a product too large for the array is refused with a clear error, and
check in a fresh process that the first call after ffg_init leaves the
device's free memory unchanged.  They need only ffg_init beforehand, so they
pass alone in a fresh process as well as after the other tests."""
import ctypes
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from oracle import limbs_to_int

pytestmark = pytest.mark.gpu


def _fn(ff):
    lib = ff.lib()
    f = lib.ffg_mul_device_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_void_p,
                  ctypes.c_size_t, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _dev(torch, x):
    return torch.from_numpy(x.view(np.int64)).cuda()


def test_no_alloc_matches_allocating_entry(ff):
    torch = pytest.importorskip("torch")
    ff.set_device(0)
    ff.init(1 << 20)
    noalloc = _fn(ff)
    rng = np.random.default_rng(99)
    for na, nb, square in ((3000, 2500, False), (700, 700, True), (40000, 40000, True)):
        a = rng.integers(0, 2**64, na, dtype=np.uint64)
        b = a if square else rng.integers(0, 2**64, nb, dtype=np.uint64)
        a[-1] |= np.uint64(1 << 63)
        b[-1] |= np.uint64(1)
        ba, bb = 64 * na, int(b[-1]).bit_length() + 64 * (nb - 1)
        da, db = _dev(torch, a), _dev(torch, b)
        want = torch.zeros(na + nb + 1, dtype=torch.int64, device="cuda")
        got = torch.full((na + nb + 1,), -1, dtype=torch.int64, device="cuda")  # every limb must be written
        torch.cuda.synchronize()
        ff.mul_device(want.data_ptr(), da.data_ptr(), na, ba, db.data_ptr(), nb, bb, square)
        rc = noalloc(got.data_ptr(), da.data_ptr(), na, ba, db.data_ptr(), nb, bb, int(square), None)
        assert rc == 0, ff.lib().ffg_last_error().decode()
        torch.cuda.synchronize()
        assert torch.equal(got, want)
        x, y = limbs_to_int(a), limbs_to_int(b)
        assert limbs_to_int(got.cpu().numpy().view(np.uint64)) == x * y


def test_no_alloc_rejects_past_its_limit(ff):
    torch = pytest.importorskip("torch")
    ff.set_device(0)
    ff.init(1 << 20)
    noalloc = _fn(ff)
    n = 300000  # a square of 300 000 limbs needs ~29 MiB of scratch
    a = torch.ones(n, dtype=torch.int64, device="cuda")
    out = torch.zeros(2 * n + 1, dtype=torch.int64, device="cuda")
    rc = noalloc(out.data_ptr(), a.data_ptr(), n, 64 * (n - 1) + 1, a.data_ptr(), n, 64 * (n - 1) + 1, 1, None)
    assert rc == 5  # FFG_E_RANGE
    assert "limit" in ff.lib().ffg_last_error().decode()


_FRESH = textwrap.dedent("""
    import ctypes, sys
    import numpy as np
    import torch
    sys.path.insert(0, sys.argv[1])
    import fastfib_b200 as ff
    ff.set_device(0)
    torch.cuda.set_device(0)
    ff.init(1 << 20)
    lib = ff.lib()
    f = lib.ffg_mul_device_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_void_p,
                  ctypes.c_size_t, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p]
    f.restype = ctypes.c_int
    n = 20000
    rng = np.random.default_rng(5)
    a = rng.integers(0, 2**64, n, dtype=np.uint64)
    a[-1] |= np.uint64(1 << 63)
    da = torch.from_numpy(a.view(np.int64)).cuda()
    out = torch.zeros(2 * n + 1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    rc = f(out.data_ptr(), da.data_ptr(), n, 64 * n, da.data_ptr(), n, 64 * n, 1, None)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    x = int.from_bytes(a.tobytes(), "little")
    ok = int.from_bytes(out.cpu().numpy().tobytes(), "little") == x * x
    print(rc, free0 - free1, int(ok))
""")


def test_no_alloc_first_call_allocates_nothing():
    """In a fresh process: ffg_init, then the first allocation-free call leaves
    the device's free memory exactly where it was (its scratch array and its
    kernels were put on the device during ffg_init) and squares exactly."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _FRESH, root], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    rc, dropped, ok = (int(v) for v in r.stdout.split()[-3:])
    assert rc == 0
    assert dropped == 0, f"device free memory fell by {dropped} bytes during the first call"
    assert ok == 1
