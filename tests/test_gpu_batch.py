"""Batched instances (one persistent launch, per-instance RKSUITE step control)
against the single-instance CPU oracle, and the split-BF16 tensor-core demag
product against FP64.

Tolerances: FP32 batch product vs oracle: 1e-5 in m at matching output times
(same FP32 arithmetic, different summation order); bf16x3: demag field within
3e-5 of the largest component against FP64, trajectories within 1e-4 in m.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MU0 = 4 * np.pi * 1e-7
GAMMA = 2.211e5


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    torch.cuda.set_device(0)
    return torch


def seeded_fields(B, seed, mag_mT=50.0):
    rng = np.random.default_rng(seed)
    ang = rng.uniform(0, 2 * np.pi, B)
    mag = rng.uniform(0, mag_mT * 1e-3, B) / MU0
    return np.stack([mag * np.cos(ang), mag * np.sin(ang), np.zeros(B)], 1)


def start_state(n, B, seed):
    rng = np.random.default_rng(seed)
    m = np.ones((B, 3, n)) / np.sqrt(3) + 0.05 * rng.standard_normal((B, 3, n))
    return m / np.linalg.norm(m, axis=1, keepdims=True)


def run_batch_vs_oracle(torch_cuda, oracle, res, L, B, precision, window, nt, atol, check_ids=None, tol=1e-6):
    from magtense_b200 import BatchSolver
    n = int(np.prod(res))
    H = seeded_fields(B, 11)
    alpha = GAMMA * np.linspace(0.02, 0.2, B)
    hext = np.zeros((B, 2, 4))
    hext[:, 1, 0] = window
    hext[:, :, 1:] = H[:, None, :]
    m0 = start_state(n, B, 12)
    t = np.linspace(0, window, nt)
    bs = BatchSolver(res, L, B, precision=precision)
    bs.assemble()
    bs.set_dynamics(hext=hext, alpha=alpha, gamma=GAMMA)
    t_out, y, flags, stats = bs.integrate(t, torch_cuda.as_tensor(m0.reshape(B, -1), device="cuda"), tol=tol)
    y = y.cpu().numpy()
    K32, _ = oracle.assemble(res, L)
    worst = 0.0
    for b in (range(B) if check_ids is None else check_ids):
        P = oracle.Problem(res, L, mode=0, gamma=GAMMA, alpha=alpha[b], hext=hext[b], K32=K32)
        to, yo, fo, so = P.solve(t, m0[b].reshape(-1), tol=tol)
        same = t_out[b] == to
        assert same.mean() > 0.9, (b, stats[b], so)
        err = np.abs(y[b][same] - yo[same]).max()
        worst = max(worst, err)
        assert err < atol, (b, err, stats[b], so)
    return worst, stats


def test_batch_fp32_matches_oracle_per_instance(torch_cuda, oracle):
    run_batch_vs_oracle(torch_cuda, oracle, [20, 5, 1], [125e-9, 31.25e-9, 3e-9], B=6, precision="fp32",
                        window=0.1e-9, nt=21, atol=1e-5)


def test_batch_fp32_many_blocks(torch_cuda, oracle):
    # 3 cell blocks x 2 instance blocks, instances checked from both blocks
    run_batch_vs_oracle(torch_cuda, oracle, [32, 10, 1], [200e-9, 62.5e-9, 3e-9], B=70, precision="fp32",
                        window=0.02e-9, nt=5, atol=1e-5, check_ids=[0, 37, 69])


@pytest.mark.parametrize("precision,rtol", [("bf16x3", 3e-5), ("bf16x2", 5e-3), ("fp16s", 1e-5)])
def test_batch_demag_split_bf16_accuracy(torch_cuda, oracle, precision, rtol):
    from magtense_b200 import BatchSolver
    res, L = [24, 8, 2], [120e-9, 40e-9, 10e-9]
    n = 384
    B = 5
    m = start_state(n, B, 3)
    bs = BatchSolver(res, L, B, precision=precision)
    bs.assemble()
    H = bs.demag_field(torch_cuda.as_tensor(m.reshape(B, -1), device="cuda")).cpu().numpy()
    P64 = oracle.Problem(res, L, mode=1)
    for b in range(B):
        Href = P64.fields(0.0, m[b])[3]
        err = np.abs(H[b] - Href).max() / np.abs(Href).max()
        assert err < rtol, (precision, b, err)


def test_batch_fp32_demag_matches_single(torch_cuda, oracle):
    from magtense_b200 import BatchSolver
    res, L = [24, 8, 2], [120e-9, 40e-9, 10e-9]
    n, B = 384, 3
    m = start_state(n, B, 4)
    bs = BatchSolver(res, L, B, precision="fp32")
    bs.assemble()
    H = bs.demag_field(torch_cuda.as_tensor(m.reshape(B, -1), device="cuda")).cpu().numpy()
    P = oracle.Problem(res, L, mode=0)
    for b in range(B):
        Href = P.fields(0.0, m[b])[3]
        assert np.abs(H[b] - Href).max() <= 1e-5 * np.abs(Href).max()


def test_batch_bf16x3_trajectories(torch_cuda, oracle):
    worst, stats = run_batch_vs_oracle(torch_cuda, oracle, [20, 5, 1], [125e-9, 31.25e-9, 3e-9], B=6,
                                       precision="bf16x3", window=0.1e-9, nt=21, atol=1e-4)
    print("bf16x3 worst |dm| vs oracle", worst)


def test_batch_fp16s_trajectories(torch_cuda, oracle):
    worst, stats = run_batch_vs_oracle(torch_cuda, oracle, [20, 5, 1], [125e-9, 31.25e-9, 3e-9], B=6,
                                       precision="fp16s", window=0.1e-9, nt=21, atol=2e-5)
    print("fp16s worst |dm| vs oracle", worst)


def test_host_streamed_trajectories_match_device(torch_cuda, monkeypatch):
    """mt_batch_integrate_host: short launches (MT_BATCH_TICKS) make the host copies of
    finished samples overlap later launches; the page-locked host trajectories equal the
    device trajectories of the same integration bit for bit, and a pageable host buffer
    is refused."""
    import ctypes
    from magtense_b200 import BatchSolver, _lib
    torch = torch_cuda
    monkeypatch.setenv("MT_BATCH_TICKS", "25")
    res, L = [20, 5, 1], [125e-9, 31.25e-9, 3e-9]
    n, B = 100, 6
    rng = np.random.default_rng(31)
    ang = rng.uniform(0, 2 * np.pi, B)
    mag = rng.uniform(5e-3, 50e-3, B) / MU0
    window = 0.05e-9
    hext = np.zeros((B, 2, 4))
    hext[:, 1, 0] = window
    hext[:, :, 1] = (mag * np.cos(ang))[:, None]
    hext[:, :, 2] = (mag * np.sin(ang))[:, None]
    m = np.ones((B, 3, n)) / np.sqrt(3) + 0.05 * rng.standard_normal((B, 3, n))
    m0 = torch.as_tensor((m / np.linalg.norm(m, axis=1, keepdims=True)).reshape(B, -1), device="cuda")
    t = np.linspace(0, window, 26)
    bs = BatchSolver(res, L, B, precision="int8")
    bs.assemble()
    bs.set_dynamics(hext=hext, alpha=GAMMA * 0.05, gamma=GAMMA)
    t_dev, y_dev, f_dev, st_dev = bs.integrate(t, m0, tol=1e-6)
    host = torch.empty((B, len(t), 3 * n), dtype=torch.float64).pin_memory()
    t_h, y_h, f_h, st_h = bs.integrate(t, m0, tol=1e-6, host_out=host)
    assert y_h is host and st_h[0]["launches"] > 3
    assert np.array_equal(t_h, t_dev) and np.array_equal(f_h, f_dev)
    assert torch.equal(host, y_dev.cpu())
    with pytest.raises(ValueError):
        bs.integrate(t, m0, tol=1e-6, host_out=torch.empty((B, len(t), 3 * n), dtype=torch.float64))
    pageable = np.zeros((B, len(t), 3 * n))
    y_tmp = torch.zeros((B, len(t), 3 * n), dtype=torch.float64, device="cuda")
    t_out = np.zeros((B, len(t)))
    flags = np.zeros((B, len(t)), dtype=np.int32)
    st = (_lib.Stats * B)()
    tc = np.zeros(1)
    rc = _lib.lib().mt_batch_integrate_host(bs._h, t.ctypes.data_as(_lib.D), len(t), ctypes.c_void_p(m0.data_ptr()),
                                            1e-6, 1e-6, tc.ctypes.data_as(_lib.D), 0, 1e-4,
                                            t_out.ctypes.data_as(_lib.D), ctypes.c_void_p(y_tmp.data_ptr()),
                                            ctypes.c_void_p(pageable.ctypes.data), flags.ctypes.data_as(_lib.I), st,
                                            ctypes.c_void_p(0))
    assert rc == -1   # MT_ERR_ARG
    bs.close()
