"""The allocation-free COO assembly entry point (v2d_assemble_coo_noalloc),
called through the C ABI, against the allocating one (v2d_assemble_coo).

It is meant for callers that cannot allocate device memory where they
assemble (a framework that owns the GPU's memory through its own pool, or a
loop that must avoid cudaMalloc/cudaFree); its scratch is a fixed array inside
the library.  Two calls in a row with different rows, states and boundary
conditions must both equal the allocating entry point bit for bit (the
tolerance the other assembly parity tests use), so nothing the first call
leaves in the shared scratch leaks into the second, and neither call may take
device memory (checked with the default memory pool's high watermark and the
free device memory).  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from cases import smooth_state

pytestmark = pytest.mark.gpu


class _PoolWatch:
    """Allocation probe: the library's stream-ordered allocations come from the
    device's default memory pool, so the pool's used-memory high watermark,
    reset just before the call, stays at the memory in use before it.  With
    check_free, the free device memory must not drop either (a plain
    cudaMalloc still held); that check is left out of a process's first call,
    where loading the library's device code maps its static data, the
    scratch array included."""

    def __init__(self, torch, check_free):
        self.check_free = check_free
        from cuda.bindings import driver as drv
        self.drv, self.torch = drv, torch
        err, self.pool = drv.cuDeviceGetDefaultMemPool(torch.cuda.current_device())
        assert err == drv.CUresult.CUDA_SUCCESS, err

    def _attr(self, a):
        err, v = self.drv.cuMemPoolGetAttribute(self.pool, a)
        assert err == self.drv.CUresult.CUDA_SUCCESS, err
        return int(v)

    def __enter__(self):
        A = self.drv.CUmemPool_attribute
        self.used0 = self._attr(A.CU_MEMPOOL_ATTR_USED_MEM_CURRENT)
        err, = self.drv.cuMemPoolSetAttribute(self.pool, A.CU_MEMPOOL_ATTR_USED_MEM_HIGH,
                                              self.drv.cuuint64_t(0))
        assert err == self.drv.CUresult.CUDA_SUCCESS, err
        self.free0 = self.torch.cuda.mem_get_info()[0]
        return self

    def __exit__(self, *exc):
        A = self.drv.CUmemPool_attribute
        self.high = self._attr(A.CU_MEMPOOL_ATTR_USED_MEM_HIGH)
        self.free1 = self.torch.cuda.mem_get_info()[0]
        return False

    def allocated_nothing(self):
        return self.high <= self.used0 and (not self.check_free or self.free1 >= self.free0)


def _call_noalloc(v2d, torch, imax, jmax, args_scalars, fields, r0, r1, maxnnz, ff_bc, ca, sa,
                  watch=False):
    from vorti2d_b200 import _lib
    dev = [torch.from_numpy(np.ascontiguousarray(f)).cuda() for f in fields]
    ptrs = (ctypes.c_void_p * 14)(*[t.data_ptr() for t in dev])
    ci = torch.zeros(maxnnz, dtype=torch.int32, device="cuda")
    cj = torch.zeros(maxnnz, dtype=torch.int32, device="cuda")
    cv = torch.zeros(maxnnz, dtype=torch.float64, device="cuda")
    b = torch.zeros(max(r1 - r0, 1), dtype=torch.float64, device="cuda")
    nnz = ctypes.c_int(-1)
    torch.cuda.synchronize()
    w = _PoolWatch(torch, watch == 2) if watch else None
    if w:
        w.__enter__()
    code = _lib.lib().v2d_assemble_coo_noalloc(
        imax, jmax, *args_scalars, ptrs, r0, r1, maxnnz, ff_bc, ca, sa, ci.data_ptr(),
        cj.data_ptr(), cv.data_ptr(), ctypes.byref(nnz), b.data_ptr(), None)
    if w:
        w.__exit__(None, None, None)
        assert w.allocated_nothing(), (w.used0, w.high, w.free0, w.free1)
    return code, nnz.value, ci.cpu().numpy(), cj.cpu().numpy(), cv.cpu().numpy(), \
        b.cpu().numpy()[:r1 - r0]


def test_noalloc_matches_allocating_entry_point_twice(v2d, oracle_mod):
    import torch
    from vorti2d_b200 import _lib
    imax, jmax = 33, 21
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    dk, de = 1.0 / (imax - 1), 1.0 / (jmax - 1)
    M = oracle_mod.core().compute_metrics(dk, de, xg, yg)
    st = smooth_state(M[8], M[9])
    N = imax * jmax
    calls = [
        # re, invdtau, inv2dt, urot, rows, ff_bc, alpha
        (80.0, 0.0, 2.5, 0.3, (0, 2 * N), 1, 0.0),
        (500.0, 1.0, 0.0, -0.2, (N // 3, N + N // 2), 2, 8.0),
    ]
    for k, (re, invdtau, inv2dt, urot, (r0, r1), ff_bc, adeg) in enumerate(calls):
        ca, sa = np.cos(np.radians(adeg)), np.sin(np.radians(adeg))
        scale = 1.0 + 0.5 * k                        # a different state on each call
        fields = [*M, *(scale * a for a in st)]
        maxnnz = 13 * (r1 - r0)
        want = v2d.core.assemble_coo(imax, jmax, re, invdtau, inv2dt, urot, dk, de, *fields,
                                     r0, r1, maxnnz, ff_bc, ca, sa)
        code, n, ci, cj, cv, b = _call_noalloc(v2d, torch, imax, jmax,
                                              (re, invdtau, inv2dt, urot, dk, de), fields,
                                              r0, r1, maxnnz, ff_bc, ca, sa,
                                              watch=1 if k == 0 else 2)
        assert code == 0, _lib.last_error()
        assert n == want[3]
        assert np.array_equal(ci[:n], want[0][:n]) and np.array_equal(cj[:n], want[1][:n])
        assert np.array_equal(cv[:n], want[2][:n])
        assert np.array_equal(b, want[4])


def test_noalloc_limits(v2d, oracle_mod):
    """A row range beyond the fixed scratch, and a maxnnz that is too small,
    are rejected with an error instead of writing anything."""
    import torch
    from vorti2d_b200 import _lib
    imax, jmax = 9, 7
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    M = oracle_mod.core().compute_metrics(1 / 8, 1 / 6, xg, yg)
    fields = [*M, *smooth_state(M[8], M[9])]
    N = imax * jmax
    code, n, *_ = _call_noalloc(v2d, torch, imax, jmax, (40.0, 0.0, 0.0, 0.0, 1 / 8, 1 / 6),
                                fields, 0, 2 * N, 10, 0, 1.0, 0.0)
    assert code == _lib.V2D_ECAPACITY and n == 0
    assert "maxnnz" in _lib.last_error()
    # a grid whose 2N rows exceed the scratch: rejected before any device work
    big = 725
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    ptrs = (ctypes.c_void_p * 14)(*([dummy.data_ptr()] * 14))
    nnz = ctypes.c_int(-1)
    code = _lib.lib().v2d_assemble_coo_noalloc(
        big, big, 40.0, 0.0, 0.0, 0.0, 1.0, 1.0, ptrs, 0, 2 * big * big, 1, 0, 1.0, 0.0,
        dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), ctypes.byref(nnz),
        dummy.data_ptr(), None)
    assert code == _lib.V2D_EARG and "scratch" in _lib.last_error()
