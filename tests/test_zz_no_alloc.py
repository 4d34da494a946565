"""The allocation-free multiply (ffg_mul_device_noalloc) against the
allocating one (ffg_mul_device), through the C ABI.

Some callers cannot allocate device memory once they are running -- work
issued while a CUDA graph is being captured, frameworks whose allocator owns
all device memory, paths that cannot afford a cudaMalloc.  This entry point
serves them from one fixed 8 MiB scratch array per GPU.  The test runs two
calls in a row (different sizes, a square and a distinct product, the
one-CTA and the four-step kernels) and requires bit-identical limbs, then
checks that a product too large for the array is refused with a clear error.
It needs only ffg_init beforehand, so it passes alone in a fresh process as
well as after the other tests."""
import ctypes

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
