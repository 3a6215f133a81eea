"""Thresholded-sparse demag (dem_appr "threshold" / "threshold_fraction";
ApplyThresholdDense, DemagAuxFunctions.f90:20-122; FindThresholdFraction :353-428;
ConvertDenseToSparse_s, util_micromag.f90:81-138) on the device, against the
oracle given the device's own FP32 tensor (so both see the same entries):

- the fraction's threshold is the oracle's bit for bit, and the kept entries are
  exactly those with |K| > threshold;
- the demag field and the right-hand side on the kept entries match the oracle's
  within 1e-5 of the largest component (FP32 sums in another order);
- an integration through MicromagProblem(demag_approx="threshold_fraction")
  matches the oracle's within 1e-5 in m;
- the reference's sparse C shims (six 1-based CSR blocks) give the product of
  the kept entries.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MU0 = 4 * np.pi * 1e-7
GAMMA = 2.211e5
BLK = [[0, 1, 2], [1, 3, 4], [2, 4, 5]]


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    torch.cuda.set_device(0)
    return torch


def rand_m(n, seed):
    rng = np.random.default_rng(seed)
    m = rng.standard_normal((3, n))
    return m / np.linalg.norm(m, axis=0)


def kept_product(K32, thr, m, Ms=8e5):
    """-Ms sum_b K_ab m_b over the entries with |K| > thr, FP64 sums of FP32 values."""
    Ks = np.where(np.abs(K32) > thr, K32, 0).astype(np.float64)
    m32 = m.astype(np.float32).astype(np.float64)
    return np.stack([-Ms * sum(Ks[BLK[a][b]] @ m32[b] for b in range(3)) for a in range(3)])


@pytest.mark.parametrize("frac", [0.5, 0.9])
def test_fraction_threshold_and_kept_entries(torch_cuda, oracle, frac):
    from magtense_b200 import Solver
    res, L = [16, 8, 2], [80e-9, 40e-9, 10e-9]
    s = Solver(res, L)
    s.assemble()
    K32 = np.ascontiguousarray(np.stack(s.get_tensor_colmajor()))
    nnz, thr = s.set_demag_threshold("threshold_fraction", frac)
    assert np.float32(thr) == np.float32(oracle.threshold_fraction(K32, frac))
    want = sum(int(np.count_nonzero(np.abs(K32[BLK[a][b]]) > thr)) for a in range(3) for b in range(3))
    assert nnz == want
    m = rand_m(s.n, 5)
    H = s.demag_field(torch_cuda.as_tensor(m.reshape(-1), device="cuda")).cpu().numpy()
    P = oracle.Problem(res, L, mode=0, K32=K32)
    P.set_threshold(thr)
    Ho = P.fields(0.0, m)[3]
    scale = np.abs(Ho).max()
    assert np.abs(H - Ho).max() <= 1e-5 * scale
    assert np.abs(H - kept_product(K32, thr, m)).max() <= 1e-5 * scale
    # the dense product differs: the threshold matters
    s.set_demag_threshold(None, 0.0)
    Hd = s.demag_field(torch_cuda.as_tensor(m.reshape(-1), device="cuda")).cpu().numpy()
    assert np.abs(Hd - H).max() > 1e-3 * scale


def test_threshold_edges(torch_cuda, oracle):
    """threshold 0 keeps every nonzero entry (the dense result); a fraction >= 1
    removes everything (no demag field)."""
    from magtense_b200 import Solver
    res, L = [10, 5, 1], [62.5e-9, 31.25e-9, 3e-9]
    s = Solver(res, L)
    s.assemble()
    m = torch_cuda.as_tensor(rand_m(s.n, 6).reshape(-1), device="cuda")
    Hd = s.demag_field(m).cpu().numpy()
    s.set_demag_threshold("threshold", 0.0)
    H0 = s.demag_field(m).cpu().numpy()
    assert np.abs(H0 - Hd).max() <= 1e-5 * np.abs(Hd).max()
    nnz, thr = s.set_demag_threshold("threshold_fraction", 1.0)
    assert nnz == 0 and thr > 1e38
    assert float(s.demag_field(m).abs().max()) == 0.0


def test_sparse_rhs_and_integration_match_oracle(torch_cuda, oracle):
    from magtense_b200 import MicromagProblem
    res, L = [20, 5, 1], [125e-9, 31.25e-9, 3e-9]
    n = 100
    h = np.array([-24.6e-3, 4.3e-3, 0.0]) / MU0
    m0 = rand_m(n, 7) + np.array([[1.0], [1.0], [1.0]])
    m0 /= np.linalg.norm(m0, axis=0)
    prob = MicromagProblem(res, L, m0=m0.T.copy(), alpha=GAMMA * 0.05, gamma=GAMMA, tol=1e-6,
                           demag_approx="threshold_fraction", dem_thres=0.8)
    t_end, nt = 0.05e-9, 11
    t_out, M, *_ = prob.run_simulation(t_end, nt, lambda t: np.tile(h, (len(t), 1)), 2)
    nnz, thr = prob.demag_sparse
    s = prob._solver_obj
    s.set_demag_threshold(None, 0.0)
    K32 = np.ascontiguousarray(np.stack(s.get_tensor_colmajor()))
    hext = np.array([[0.0, *h], [t_end, *h]])
    P = oracle.Problem(res, L, mode=0, gamma=GAMMA, alpha=GAMMA * 0.05, hext=hext, K32=K32)
    P.set_threshold(thr)
    # right-hand side at the start state
    s.set_demag_threshold("threshold", thr)
    s.set_dynamics(solver=2, gamma=GAMMA, alpha=GAMMA * 0.05, hext=hext)
    d = s.rhs(0.0, torch_cuda.as_tensor(m0.reshape(-1), device="cuda")).cpu().numpy()
    dref = P.rhs(0.0, m0.reshape(-1))
    assert np.abs(d - dref).max() <= 1e-5 * np.abs(dref).max()
    to, yo, _, so = P.solve(np.linspace(0, t_end, nt), m0.reshape(-1), tol=1e-6)
    got = M[:, :, 0, :].transpose(0, 2, 1).reshape(nt, -1)
    same = t_out == to
    assert same.mean() > 0.9
    assert np.abs(got[same] - yo[same]).max() < 1e-5


def test_reference_sparse_shims(torch_cuda, oracle):
    """icl_initDemagMatrices_sparse six times (1-based CSR of each block, rowInds[n]
    = nnz + rowInds[0]), then icl_MVMult_GetH_sparse: H = pref * K * M."""
    from magtense_b200 import Solver, _lib
    res, L = [12, 6, 1], [60e-9, 30e-9, 3e-9]
    s = Solver(res, L)
    s.assemble()
    K32 = np.ascontiguousarray(np.stack(s.get_tensor_colmajor()))
    n = s.n
    thr = np.float32(np.quantile(np.abs(K32[K32 != 0]), 0.7))
    lib = _lib.lib()
    IP, FP = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float)
    keep = []
    for c in range(6):
        rows, cols, vals = [1], [], []
        for i in range(n):
            js = np.nonzero(np.abs(K32[c][i]) > thr)[0]
            cols.extend((js + 1).tolist())
            vals.extend(K32[c][i][js].tolist())
            rows.append(rows[-1] + len(js))
        r = np.array(rows, dtype=np.int32)
        cc = np.array(cols if cols else [1], dtype=np.int32)
        v = np.array(vals if vals else [0.0], dtype=np.float32)
        keep.append((r, cc, v))
        rc = lib.icl_initDemagMatrices_sparse(ctypes.byref(ctypes.c_int(n)), ctypes.byref(ctypes.c_int(len(cols))),
                                              ctypes.byref(ctypes.c_int(c + 1)), v.ctypes.data_as(FP),
                                              cc.ctypes.data_as(IP), r.ctypes.data_as(IP))
        assert rc == 0, lib.mt_last_error()
    m = rand_m(n, 9).astype(np.float32)
    H = [np.zeros(n, dtype=np.float32) for _ in range(3)]
    pref = ctypes.c_float(-1.0)
    rc = lib.icl_MVMult_GetH_sparse(*(x.ctypes.data_as(FP) for x in m), *(x.ctypes.data_as(FP) for x in H),
                                    ctypes.byref(ctypes.c_int(n)), ctypes.byref(pref))
    assert rc == 0, lib.mt_last_error()
    want = kept_product(K32, thr, m.astype(np.float64), Ms=1.0)
    got = np.stack(H).astype(np.float64)
    assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()
    assert lib.icl_destroy() == 0
