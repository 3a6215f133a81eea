"""The exact fixed-point demag product ("int8": tcgen05 kind::i8, twelve limb
products accumulated exactly) against the oracle's restatement of the same
definition (oracle mode 2), both given the FP32 tensor the device assembled
(device and host FP64 libm may differ in the last bit, so the two assemblies
agree to 2 FP32 ulp only).  The product is exact, so the demag field must
match the oracle bit for bit, whatever the Stream-K split of the k range; the
whole right-hand side then matches too, and so do the per-instance RKSUITE
trajectories.  Accuracy against the FP64 tensor and product: 2e-5 of the
largest component (32-bit fixed-point tensor rows; the FP32 tensor the rows
are made from carries most of it)."""
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


def unit_states(n, B, seed, tilt=0.05):
    rng = np.random.default_rng(seed)
    m = np.ones((B, 3, n)) / np.sqrt(3) + tilt * rng.standard_normal((B, 3, n))
    return m / np.linalg.norm(m, axis=1, keepdims=True)


def device_tensor(res, L):
    """The FP32 tensor as the device assembles it, in the oracle's [c][i][j] layout."""
    from magtense_b200 import Solver
    s = Solver(res, L)
    s.assemble()
    K = np.ascontiguousarray(np.stack(s.get_tensor_colmajor()))
    s.close()
    return K


def demag_batch(torch_cuda, res, L, m):
    from magtense_b200 import BatchSolver
    B = m.shape[0]
    bs = BatchSolver(res, L, B, precision="int8")
    bs.assemble()
    H = bs.demag_field(torch_cuda.as_tensor(m.reshape(B, -1), device="cuda")).cpu().numpy()
    bs.close()
    return H.reshape(B, -1)


def test_int8_demag_bit_exact_small(torch_cuda, oracle):
    res, L = [24, 8, 2], [120e-9, 40e-9, 10e-9]
    n, B = 384, 5
    m = unit_states(n, B, 3, tilt=1.0)
    H = demag_batch(torch_cuda, res, L, m)
    P2 = oracle.Problem(res, L, mode=2, K32=device_tensor(res, L))
    P64 = oracle.Problem(res, L, mode=1)
    for b in range(B):
        Hq = P2.fields(0.0, m[b])[3].reshape(-1)
        assert np.array_equal(H[b], Hq), (b, np.abs(H[b] - Hq).max())
        H64 = P64.fields(0.0, m[b])[3].reshape(-1)
        assert np.abs(H[b] - H64).max() <= 2e-5 * np.abs(H64).max()


@pytest.mark.parametrize("res,L,B", [
    # film of 1600 cells, 200 instances: 4 instance tiles x 39 row blocks x 78 k steps over all SMs,
    # so most tiles are summed from several CTA segments
    ([80, 20, 1], [500e-9, 125e-9, 3e-9], 200),
    # fewer units than SMs: every unit on its own CTA, each tile summed from six segments
    ([20, 5, 1], [125e-9, 31.25e-9, 3e-9], 2),
])
def test_int8_demag_bit_exact_streamk_segments(torch_cuda, oracle, res, L, B):
    n = int(np.prod(res))
    m = unit_states(n, B, 5, tilt=0.3)
    H = demag_batch(torch_cuda, res, L, m)
    P2 = oracle.Problem(res, L, mode=2, K32=device_tensor(res, L))
    for b in sorted({0, min(63, B - 1), min(64, B - 1), B // 2, B - 1}):
        Hq = P2.fields(0.0, m[b])[3].reshape(-1)
        assert np.array_equal(H[b], Hq), (b, np.abs(H[b] - Hq).max())


def test_int8_demag_exact_linearity(torch_cuda):
    # on the 2^-30 grid the fixed-point product is exactly linear: H_int(a + c) = H_int(a) + H_int(c)
    res, L = [40, 10, 1], [250e-9, 62.5e-9, 3e-9]
    n = 400
    rng = np.random.default_rng(9)
    a = np.round(rng.uniform(-0.9, 0.9, (1, 3, n)) * 2.0**30) / 2.0**30
    c = np.round(rng.uniform(-0.9, 0.9, (1, 3, n)) * 2.0**30) / 2.0**30
    m = np.concatenate([a, c, a + c], 0)
    H = demag_batch(torch_cuda, res, L, m)
    # -Ms 2^k H_int rounds once per field, so the sum agrees to one rounding of the largest value
    assert np.abs(H[2] - (H[0] + H[1])).max() <= 1e-12 * np.abs(H[2]).max()


def test_int8_range_error(torch_cuda):
    from magtense_b200 import BatchSolver
    from magtense_b200._lib import MTError
    res, L = [8, 4, 1], [40e-9, 20e-9, 3e-9]
    bs = BatchSolver(res, L, 2, precision="int8")
    bs.assemble()
    m = np.zeros((2, 3 * 32))
    m[1, 5] = 2.5
    with pytest.raises(MTError):
        bs.demag_field(torch_cuda.as_tensor(m, device="cuda"))
    bs.close()


def test_int8_trajectories_match_oracle(torch_cuda, oracle):
    from magtense_b200 import BatchSolver
    res, L = [20, 5, 1], [125e-9, 31.25e-9, 3e-9]
    n, B = 100, 6
    rng = np.random.default_rng(11)
    ang = rng.uniform(0, 2 * np.pi, B)
    mag = rng.uniform(0, 50e-3, B) / MU0
    Hf = np.stack([mag * np.cos(ang), mag * np.sin(ang), np.zeros(B)], 1)
    window = 0.1e-9
    alpha = GAMMA * np.linspace(0.02, 0.2, B)
    hext = np.zeros((B, 2, 4))
    hext[:, 1, 0] = window
    hext[:, :, 1:] = Hf[:, None, :]
    m0 = unit_states(n, B, 12)
    t = np.linspace(0, window, 21)
    bs = BatchSolver(res, L, B, precision="int8")
    bs.assemble()
    bs.set_dynamics(hext=hext, alpha=alpha, gamma=GAMMA)
    t_out, y, flags, stats = bs.integrate(t, torch_cuda.as_tensor(m0.reshape(B, -1), device="cuda"), tol=1e-6)
    y = y.cpu().numpy()
    K32 = device_tensor(res, L)
    for b in range(B):
        P = oracle.Problem(res, L, mode=2, gamma=GAMMA, alpha=alpha[b], hext=hext[b], K32=K32)
        to, yo, fo, so = P.solve(t, m0[b].reshape(-1), tol=1e-6)
        assert np.array_equal(t_out[b], to), (b, stats[b], so)
        assert stats[b]["f_evals"] == so["f_evals"], (b, stats[b], so)
        assert np.array_equal(y[b], yo), (b, np.abs(y[b] - yo).max())
    bs.close()


def test_micromag_run_batch_matches_oracle(torch_cuda, oracle):
    """MicromagProblem.run_batch: per-instance constant fields, damping and initial
    states on the int8 batched path, each instance bit-exact with the oracle's
    single-instance run of the same definition, in the reference's M layout."""
    from magtense_b200 import MicromagProblem
    res, L = [20, 5, 1], [125e-9, 31.25e-9, 3e-9]
    n, B = 100, 3
    m0 = unit_states(n, B, 21)                                  # (B, 3, n)
    rng = np.random.default_rng(22)
    Hf = np.stack([rng.uniform(-30e-3, 30e-3, B) / MU0, rng.uniform(-30e-3, 30e-3, B) / MU0, np.zeros(B)], 1)
    alpha = GAMMA * np.array([0.02, 0.1, 0.5])
    prob = MicromagProblem(res, L, gamma=GAMMA, alpha=GAMMA * 0.02, tol=1e-6)
    t_end, nt = 0.05e-9, 11
    t_out, M, pts = prob.run_batch(t_end, nt, Hf, m0=m0.transpose(0, 2, 1), alpha=alpha)
    assert M.shape == (B, nt, n, 1, 3) and pts.shape == (n, 3)
    K32 = device_tensor(res, L)
    t = np.linspace(0, t_end, nt)
    for b in range(B):
        hext = np.array([[0.0, *Hf[b]], [t_end, *Hf[b]]])
        P = oracle.Problem(res, L, mode=2, gamma=GAMMA, alpha=alpha[b], hext=hext, K32=K32)
        to, yo, _, so = P.solve(t, m0[b].reshape(-1), tol=1e-6)
        assert np.array_equal(t_out[b], to), b
        assert prob.last_stats[b]["f_evals"] == so["f_evals"], (b, prob.last_stats[b], so)
        assert np.array_equal(M[b, :, :, 0, :].transpose(0, 2, 1).reshape(nt, -1), yo), b


def test_std_prob_4_dataset_sequences_match_oracle(torch_cuda, oracle, tmp_path):
    """The dataset driver: a short relaxation from the reference's s-state recipe,
    then three seeded sequences in one batched run; each sequence equals the
    oracle's single-instance run of the same definition, bit for bit, in the
    database layout."""
    from magtense_b200 import dataset as D
    res, L = (16, 8, 1), (100e-9, 50e-9, 3e-9)
    n = 128
    st = D.s_state(res, L, t_end=2e-9, nt=5, nt_h_ext=50)
    assert st.shape == (n, 3) and np.all(np.isfinite(st))
    fields = D.std_prob_4_fields(3, seed=5)
    t_steps, dt = 8, 4e-12
    seq, stats = D.std_prob_4_sequences(st, res, fields, L, t_steps, dt, precision="int8")
    assert seq.shape == (3, t_steps, 3, 16, 8) and seq.dtype == np.float32
    K32 = device_tensor(list(res), list(L))
    t = np.linspace(0, dt * t_steps, t_steps)
    m0 = np.concatenate((st[:, 0], st[:, 1], st[:, 2]))
    for b in range(3):
        h = fields[b] / 1000 / MU0
        P = oracle.Problem(list(res), list(L), mode=2, gamma=D.GAMMA, alpha=D.ALPHA,
                           hext=np.array([[0.0, *h], [dt * t_steps, *h]]), K32=K32)
        _, yo, _, so = P.solve(t, m0, tol=1e-4)
        want = D.sequence_layout(yo.reshape(t_steps, 3, n).transpose(0, 2, 1), res).astype(np.float32)
        assert stats[b]["f_evals"] == so["f_evals"], (b, stats[b], so)
        assert np.array_equal(seq[b], want), b
    out = D.write_database(tmp_path / "db", seq, fields, (0, 3))
    assert out.exists()


def test_gemm_schedules_are_bit_exact_and_tuned(torch_cuda, oracle):
    """The autotuner's candidate schedules of the int8 product (Stream-K CTA count from
    all SMs down to two thirds of them, tile-major or row-major unit order) all give
    the same bits, equal to oracle mode 2; the tuned schedule is one of them."""
    from magtense_b200 import BatchSolver, MTError
    res, L = [24, 8, 2], [120e-9, 40e-9, 10e-9]
    n, B = 384, 192
    m = unit_states(n, B, 17, tilt=1.0).reshape(B, -1)
    bs = BatchSolver(res, L, B, precision="int8")
    bs.assemble()
    mt = torch_cuda.as_tensor(m, device="cuda")
    H0 = bs.demag_field(mt).cpu().numpy().reshape(B, -1)
    tiles = len(bs.schedule())
    sms = torch_cuda.cuda.get_device_properties(0).multi_processor_count
    lo = max(1, 2 * sms // 3)
    for G, order in [(sms, 0), (sms, 1), (lo, 0), (lo, 1), (sms - 8, 1), (lo + 5, 0)]:
        bs.set_schedule([(G, order)] * tiles)
        H = bs.demag_field(mt).cpu().numpy().reshape(B, -1)
        assert np.array_equal(H, H0), (G, order)
    with pytest.raises(MTError):
        bs.set_schedule([(lo - 1, 0)] * tiles)
    sched = bs.tune()
    assert len(sched) == tiles
    for k, G, order in sched:
        assert lo <= G <= sms and order in ("tile-major", "row-major")
    H = bs.demag_field(mt).cpu().numpy().reshape(B, -1)
    assert np.array_equal(H, H0)
    P2 = oracle.Problem(res, L, mode=2, K32=device_tensor(res, L))
    for b in (0, 77, 191):
        Hm = P2.fields(0.0, m[b])[3].reshape(-1)
        assert np.array_equal(H0[b], Hm), b
    bs.close()


def test_every_instance_owned_when_blocks_split_unevenly(torch_cuda):
    """300 film instances (n = 1600): 13 x 3 tiles, so 148 SMs would allow three splits
    of each 128-instance block; the splits must divide the block (two here), or the
    last instances of every block have no coroutine owner.  Instances at the ends of
    the blocks follow the same bits as the same instances integrated in a small batch
    (the exact product makes every instance independent of the others)."""
    from magtense_b200 import BatchSolver
    res, L = [80, 20, 1], [500e-9, 125e-9, 3e-9]
    n, B = 1600, 300
    rng = np.random.default_rng(21)
    ang = rng.uniform(0, 2 * np.pi, B)
    mag = rng.uniform(5e-3, 50e-3, B) / MU0
    Hf = np.stack([mag * np.cos(ang), mag * np.sin(ang), np.zeros(B)], 1)
    window = 0.002e-9
    hext = np.zeros((B, 2, 4))
    hext[:, 1, 0] = window
    hext[:, :, 1:] = Hf[:, None, :]
    m0 = unit_states(n, B, 22)
    t = np.linspace(0, window, 3)
    bs = BatchSolver(res, L, B, precision="int8")
    bs.assemble()
    bs.set_dynamics(hext=hext, alpha=GAMMA * 0.02, gamma=GAMMA)
    t_out, y, _, stats = bs.integrate(t, torch_cuda.as_tensor(m0.reshape(B, -1), device="cuda"), tol=1e-6)
    y = y.cpu().numpy()
    bs.close()
    assert all(s["f_evals"] > 0 and s["status"] == 0 for s in stats)
    pick = [0, 126, 127, 255, 299]
    sb = BatchSolver(res, L, len(pick), precision="int8")
    sb.assemble()
    sb.set_dynamics(hext=hext[pick], alpha=GAMMA * 0.02, gamma=GAMMA)
    t2, y2, _, st2 = sb.integrate(t, torch_cuda.as_tensor(m0[pick].reshape(len(pick), -1), device="cuda"), tol=1e-6)
    y2 = y2.cpu().numpy()
    sb.close()
    for k, b in enumerate(pick):
        assert stats[b]["f_evals"] == st2[k]["f_evals"], (b, stats[b], st2[k])
        assert np.array_equal(t_out[b], t2[k]) and np.array_equal(y[b], y2[k]), b
