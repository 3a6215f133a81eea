"""mt_rhs_noalloc: the allocation-free right-hand side, for callers that may not
allocate device memory (a host framework that hands out all device memory from
its own pool, or a host program whose device-memory budget is fixed once it has
started).  Its scratch is a fixed array inside the library, so the call itself
allocates nothing.

Checked through the C ABI against mt_rhs on two calls in a row (the array keeps
the previous call's contents, which must not leak into the next result), on a
handle whose first right-hand side is the allocation-free one (device free
memory unchanged across its calls), and the grid-size limit.  Collected last so
that a stop at the first failure has already run every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MU0 = 4 * np.pi * 1e-7


def test_noalloc_rhs_matches_rhs_twice():
    import torch
    from magtense_b200 import Solver, _lib
    torch.cuda.set_device(0)
    res, L = [24, 10, 2], [150e-9, 62.5e-9, 6e-9]
    n = 480
    rng = np.random.default_rng(21)
    u = rng.standard_normal((n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    s = Solver(res, L, K0=4e3, u_ea=u)
    s.assemble()
    hext = np.array([[0.0, 2e4, -1e4, 5e3], [1e-9, -2e4, 1e4, 0.0]])
    s.set_dynamics(solver=2, gamma=2.211e5, alpha=2.211e5 * 0.05, hext=hext)
    lib = _lib.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call, seed in enumerate((1, 2)):
        m = rng.standard_normal((3, n)) + (0.5 if seed == 2 else 0.0)
        m = torch.as_tensor((m / np.linalg.norm(m, axis=0)).reshape(-1), device="cuda")
        t = 0.2e-9 * (call + 1)
        ref = torch.empty(3 * n, dtype=torch.float64, device="cuda")
        got = torch.full((3 * n,), float("nan"), dtype=torch.float64, device="cuda")
        _lib.check(lib.mt_rhs(s._h, t, ctypes.c_void_p(m.data_ptr()), ctypes.c_void_p(ref.data_ptr()), stream),
                   "mt_rhs")
        _lib.check(lib.mt_rhs_noalloc(s._h, t, ctypes.c_void_p(m.data_ptr()), ctypes.c_void_p(got.data_ptr()),
                                      stream), "mt_rhs_noalloc")
        torch.cuda.synchronize()
        r, g = ref.cpu().numpy(), got.cpu().numpy()
        assert np.all(np.isfinite(g))
        np.testing.assert_allclose(g, r, rtol=1e-12, atol=1e-12 * np.abs(r).max())


def test_noalloc_first_on_a_fresh_handle_allocates_nothing():
    """The handle has never run mt_rhs (so it holds no FP32 copy of m of its own):
    the first call sets up the array's address, later calls leave the device's free
    memory as it was, and the result equals mt_rhs."""
    import torch
    from magtense_b200 import Solver, _lib
    torch.cuda.set_device(0)
    res, L = [20, 5, 1], [125e-9, 31.25e-9, 3e-9]
    n = 100
    s = Solver(res, L)
    s.assemble()
    s.set_dynamics(solver=2, gamma=2.211e5, alpha=2.211e5 * 0.02,
                   hext=np.array([[0.0, -2e4, 3e3, 0.0], [1e-9, -2e4, 3e3, 0.0]]))
    lib = _lib.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(5)
    ms = []
    for _ in range(3):
        m = rng.standard_normal((3, n))
        ms.append(torch.as_tensor((m / np.linalg.norm(m, axis=0)).reshape(-1), device="cuda"))
    outs = [torch.full((3 * n,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(3)]
    refs = [torch.empty(3 * n, dtype=torch.float64, device="cuda") for _ in range(3)]
    _lib.check(lib.mt_rhs_noalloc(s._h, 0.1e-9, ctypes.c_void_p(ms[0].data_ptr()),
                                  ctypes.c_void_p(outs[0].data_ptr()), stream), "mt_rhs_noalloc")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for k in (1, 2):
        _lib.check(lib.mt_rhs_noalloc(s._h, 0.1e-9 * (k + 1), ctypes.c_void_p(ms[k].data_ptr()),
                                      ctypes.c_void_p(outs[k].data_ptr()), stream), "mt_rhs_noalloc")
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    for k in range(3):
        _lib.check(lib.mt_rhs(s._h, 0.1e-9 * (k + 1), ctypes.c_void_p(ms[k].data_ptr()),
                              ctypes.c_void_p(refs[k].data_ptr()), stream), "mt_rhs")
    torch.cuda.synchronize()
    for k in range(3):
        r, g = refs[k].cpu().numpy(), outs[k].cpu().numpy()
        assert np.all(np.isfinite(g))
        np.testing.assert_allclose(g, r, rtol=1e-12, atol=1e-12 * np.abs(r).max())


def test_noalloc_rejects_oversized_grid():
    import torch
    from magtense_b200 import _lib
    torch.cuda.set_device(0)
    lib = _lib.lib()
    g = _lib.Grid(200, 100, 1, 1e-6, 5e-7, 3e-9)          # 20000 cells > 16384
    h = ctypes.c_void_p()
    _lib.check(lib.mt_create(ctypes.byref(g), ctypes.byref(h)), "mt_create")
    try:
        rc = lib.mt_rhs_noalloc(h, 0.0, ctypes.c_void_p(0), ctypes.c_void_p(0), ctypes.c_void_p(0))
        assert rc == -1
        assert b"16384" in lib.mt_last_error()
    finally:
        lib.mt_destroy(h)
