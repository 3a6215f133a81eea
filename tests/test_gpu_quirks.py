"""Reference behaviours on the device path, each against the oracle:

* the damping table: alpha0 = 0 selects interp1 of the alpha(t) table
  (alpha(), LandauLifshitzEquationSolver.f90:281-294), on the single-instance
  path (FP32 product, oracle mode 0, within 1e-5 in m) and on the batched int8
  path (oracle mode 2, bit for bit);
* the convergence exit: at a time of t_conv the run stops once
  max|y - y_last| < conv_tol and stores that state
  (MagTense_ODE_RKSuite, ODE_Solvers.f90:210-222), on both paths;
* a 32x32x4 grid (nz > 1, exchange along z, uniaxial anisotropy, the large
  configuration's material) over more than 50 evaluations;
* three films of the ragged set, integrated together in one ragged launch;
* explicit (quasi-static) field branches on the batched path: each instance
  takes its fields in turn from the state the previous one ended in
  (LandauLifshitzEquationSolver.f90:136-186), with the convergence exit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MU0 = 4 * np.pi * 1e-7
GAMMA = 2.211e5
FILM = ([20, 5, 1], [125e-9, 31.25e-9, 3e-9])


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
    from magtense_b200 import Solver
    s = Solver(res, L)
    s.assemble()
    K = np.ascontiguousarray(np.stack(s.get_tensor_colmajor()))
    s.close()
    return K


def matched_error(t_g, y_g, t_r, y_r, min_matched=0.9):
    """Largest difference over the samples both runs took at the same time (a flag-3
    return every 5000 evaluations moves a sample to the internal time)."""
    same = np.asarray(t_g) == np.asarray(t_r)
    assert same.mean() >= min_matched, same.mean()
    return float(np.abs(np.asarray(y_g)[same] - np.asarray(y_r)[same]).max())


# a damping table that falls from alpha_G = 0.5 to 0.02 over the first 0.06 ns
ALPHA_TAB = np.array([[0.0, GAMMA * 0.5], [0.02e-9, GAMMA * 0.3], [0.06e-9, GAMMA * 0.02], [1e-9, GAMMA * 0.02]])


def test_alpha_table_single_instance(torch_cuda, oracle):
    from magtense_b200 import Solver
    res, L = FILM
    n = 100
    h = np.array([-24.6e-3, 4.3e-3, 0.0]) / MU0
    hext = np.array([[0.0, *h], [1e-9, *h]])
    s = Solver(res, L)
    s.assemble()
    s.set_dynamics(solver=2, gamma=GAMMA, alpha=0.0, alpha_tab=ALPHA_TAB, hext=hext)
    P = oracle.Problem(res, L, mode=0, gamma=GAMMA, alpha=0.0, alpha_tab=ALPHA_TAB, hext=hext)
    m0 = unit_states(n, 1, 31)[0].reshape(-1)
    t = np.linspace(0, 0.1e-9, 21)
    t_g, y_g, _, st = s.integrate(t, torch_cuda.as_tensor(m0, device="cuda"), tol=1e-6)
    t_r, y_r, _, so = P.solve(t, m0, tol=1e-6)
    err = matched_error(t_g, y_g.cpu().numpy(), t_r, y_r)
    assert err < 1e-5, (err, st, so)
    # the table matters: a constant alpha_G = 0.02 gives another trajectory
    s.set_dynamics(solver=2, gamma=GAMMA, alpha=GAMMA * 0.02, hext=hext)
    _, y_c, _, _ = s.integrate(t, torch_cuda.as_tensor(m0, device="cuda"), tol=1e-6)
    assert float((y_c - y_g).abs().max()) > 1e-2


def test_alpha_table_batched_int8_bit_exact(torch_cuda, oracle):
    """Instances with alpha 0 follow the table, the others their own constant."""
    from magtense_b200 import MicromagProblem
    res, L = FILM
    n, B = 100, 3
    m0 = unit_states(n, B, 32)
    rng = np.random.default_rng(33)
    Hf = np.stack([rng.uniform(-30e-3, 30e-3, B) / MU0, rng.uniform(-30e-3, 30e-3, B) / MU0, np.zeros(B)], 1)
    alpha = np.array([0.0, GAMMA * 0.1, 0.0])
    prob = MicromagProblem(res, L, gamma=GAMMA, alpha=0.0, tol=1e-6, t_alpha=ALPHA_TAB[:, 0],
                           alpha_fct=lambda t: np.interp(t, ALPHA_TAB[:, 0], ALPHA_TAB[:, 1]))
    t_end, nt = 0.05e-9, 11
    t_out, M, _ = prob.run_batch(t_end, nt, Hf, m0=m0.transpose(0, 2, 1), alpha=alpha)
    K32 = device_tensor(res, L)
    t = np.linspace(0, t_end, nt)
    for b in range(B):
        hext = np.array([[0.0, *Hf[b]], [t_end, *Hf[b]]])
        P = oracle.Problem(res, L, mode=2, gamma=GAMMA, alpha=alpha[b], alpha_tab=prob.alphat, hext=hext, K32=K32)
        to, yo, _, so = P.solve(t, m0[b].reshape(-1), tol=1e-6)
        assert np.array_equal(t_out[b], to), b
        assert prob.last_stats[b]["f_evals"] == so["f_evals"], (b, prob.last_stats[b], so)
        assert np.array_equal(M[b, :, :, 0, :].transpose(0, 2, 1).reshape(nt, -1), yo), b


def relax_case():
    """Damped relaxation (alpha_G = 1, zero field) checked for convergence at every output."""
    res, L = FILM
    t = np.linspace(0, 0.4e-9, 41)
    return res, L, t, t[1:], 2e-3


def test_convergence_exit_single_instance(torch_cuda, oracle):
    from magtense_b200 import Solver
    res, L, t, t_conv, conv_tol = relax_case()
    n = 100
    m0 = unit_states(n, 1, 41, tilt=0.3)[0].reshape(-1)
    s = Solver(res, L)
    s.assemble()
    zero = np.array([[0.0, 0.0, 0.0, 0.0], [1e-9, 0.0, 0.0, 0.0]])
    s.set_dynamics(solver=2, gamma=GAMMA, alpha=GAMMA * 1.0, hext=zero)
    t_g, y_g, f_g, st = s.integrate(t, torch_cuda.as_tensor(m0, device="cuda"), tol=1e-6, t_conv=t_conv,
                                    conv_tol=conv_tol)
    P = oracle.Problem(res, L, mode=0, gamma=GAMMA, alpha=GAMMA * 1.0, hext=zero)
    t_r, y_r, f_r, so = P.solve(t, m0, tol=1e-6, t_conv=t_conv, conv_tol=conv_tol)
    k = st["converged_at"]
    assert 0 < k < len(t) - 1, (st, so)          # the exit happened before the last output
    assert k == so["converged_at"], (st, so)
    assert np.array_equal(t_g[:k + 1], t_r[:k + 1])
    assert np.abs(y_g.cpu().numpy()[:k + 1] - y_r[:k + 1]).max() < 1e-5
    assert float(y_g[k + 1:].abs().max()) == 0.0 and np.abs(y_r[k + 1:]).max() == 0.0   # never written


def test_convergence_exit_batched_int8_bit_exact(torch_cuda, oracle):
    from magtense_b200 import BatchSolver
    res, L, t, t_conv, _ = relax_case()
    n, B = 100, 4
    m0 = unit_states(n, B, 42, tilt=0.3)
    conv_tol = 2e-3
    alpha = GAMMA * np.array([1.0, 0.5, 1.0, 0.05])
    hext = np.zeros((B, 2, 4))
    hext[:, 1, 0] = 1e-9
    hext[3, :, 1] = 5e3
    bs = BatchSolver(res, L, B, precision="int8")
    bs.assemble()
    bs.set_dynamics(hext=hext, alpha=alpha, gamma=GAMMA)
    t_out, y, flags, stats = bs.integrate(t, torch_cuda.as_tensor(m0.reshape(B, -1), device="cuda"), tol=1e-6,
                                          t_conv=t_conv, conv_tol=conv_tol)
    y = y.cpu().numpy()
    K32 = device_tensor(res, L)
    exits = 0
    for b in range(B):
        P = oracle.Problem(res, L, mode=2, gamma=GAMMA, alpha=alpha[b], hext=hext[b], K32=K32)
        to, yo, _, so = P.solve(t, m0[b].reshape(-1), tol=1e-6, t_conv=t_conv, conv_tol=conv_tol)
        assert stats[b]["converged_at"] == so["converged_at"], (b, stats[b], so)
        assert stats[b]["f_evals"] == so["f_evals"], (b, stats[b], so)
        k = so["converged_at"]
        upto = (k + 1) if k >= 0 else len(t)
        assert np.array_equal(t_out[b][:upto], to[:upto]), b
        assert np.array_equal(y[b][:upto], yo[:upto]), b
        exits += k >= 0
    assert exits >= 2
    bs.close()


def test_32x32x4_anisotropic_trajectory(torch_cuda, oracle):
    """The large configuration's physics on a grid the oracle integrates quickly:
    5 nm cubes with nz = 4, K = 5e3 J/m^3 along a seeded axis, 10 mT, alpha_G = 0.1,
    seeded random unit m0."""
    from magtense_b200 import Solver
    res, L = [32, 32, 4], [160e-9, 160e-9, 20e-9]
    n = 4096
    rng = np.random.default_rng(1)
    axis = rng.standard_normal(3)
    axis /= np.linalg.norm(axis)
    u = np.tile(axis, (n, 1))
    m = rng.standard_normal((3, n))
    m0 = (m / np.linalg.norm(m, axis=0)).reshape(-1)
    h = np.array([10e-3 / MU0, 0.0, 0.0])
    win = 0.002e-9
    hext = np.array([[0.0, *h], [win, *h]])
    s = Solver(res, L, K0=5e3, u_ea=u)
    s.assemble()
    s.set_dynamics(solver=2, gamma=GAMMA, alpha=GAMMA * 0.1, hext=hext)
    t = np.linspace(0, win, 5)
    t_g, y_g, _, st = s.integrate(t, torch_cuda.as_tensor(m0, device="cuda"), tol=1e-6)
    assert st["f_evals"] >= 50, st
    P = oracle.Problem(res, L, mode=0, K0=5e3, u_ea=u, gamma=GAMMA, alpha=GAMMA * 0.1, hext=hext,
                       K32=np.ascontiguousarray(np.stack(s.get_tensor_colmajor())))
    t_r, y_r, _, so = P.solve(t, m0, tol=1e-6)
    err = matched_error(t_g, y_g.cpu().numpy(), t_r, y_r, min_matched=1.0)
    print(f"32x32x4: {st['f_evals']} evaluations (oracle {so['f_evals']}), max |m_gpu - m_oracle| {err:.2e}")
    assert err < 1e-5, (err, st, so)
    # the two FP32 products round differently, which moves RKSUITE's step choices at tol 1e-6
    assert abs(st["f_evals"] - so["f_evals"]) <= 0.3 * max(st["f_evals"], so["f_evals"])


def test_ragged_instances_match_oracle(torch_cuda, oracle):
    """Films of the ragged configuration (nx from the seeded draw U{20..120}, seed 2,
    ny = nx/4, 6.25 x 6.25 x 3 nm cells) in one ragged launch; the three smallest
    against the oracle."""
    from magtense_b200 import Solver, integrate_ragged
    nxs = np.random.default_rng(2).integers(20, 121, 64)[:8]
    rng = np.random.default_rng(51)
    probs = []
    for nx in nxs:
        nx = int(nx)
        ny = nx // 4
        res, L = (nx, ny, 1), (nx * 6.25e-9, ny * 6.25e-9, 3e-9)
        ang, mag = rng.uniform(0, 2 * np.pi), rng.uniform(0, 50e-3) / MU0
        h = np.array([mag * np.cos(ang), mag * np.sin(ang), 0.0])
        hext = np.array([[0.0, *h], [1e-9, *h]])
        sv = Solver(res, L)
        sv.assemble()
        sv.set_dynamics(solver=2, gamma=GAMMA, alpha=GAMMA * 0.02, hext=hext)
        probs.append((sv, unit_states(nx * ny, 1, int(nx))[0].reshape(-1), res, L, hext))
    t = np.linspace(0, 0.02e-9, 11)
    t_out, ys, _, st = integrate_ragged([p[0] for p in probs], t, [p[1] for p in probs], tol=1e-6, graph=True)
    for k in np.argsort([p[0].n for p in probs])[:3]:
        sv, m0, res, L, hext = probs[k]
        P = oracle.Problem(res, L, mode=0, gamma=GAMMA, alpha=GAMMA * 0.02, hext=hext,
                           K32=np.ascontiguousarray(np.stack(sv.get_tensor_colmajor())))
        to, yo, _, so = P.solve(t, m0, tol=1e-6)
        err = matched_error(t_out[k], ys[k].cpu().numpy(), to, yo)
        assert err < 1e-5, (k, res, err, st[k], so)
        assert abs(st[k]["f_evals"] - so["f_evals"]) <= 0.3 * max(st[k]["f_evals"], so["f_evals"]), (st[k], so)


def test_explicit_branches_batched_bit_exact(torch_cuda, oracle):
    """Three hysteresis branches (instances) of three quasi-static fields each, with
    the convergence exit; every branch equals the oracle's explicit run with its
    field rows taken in turn, chained from the sample each run ended with."""
    from magtense_b200 import MicromagProblem
    res, L = FILM
    n, B, K = 100, 3, 3
    m0 = unit_states(n, B, 61, tilt=0.2)
    fields = np.zeros((B, K, 3))
    fields[:, :, 0] = np.array([[40e-3, 0.0, -40e-3], [-20e-3, 20e-3, 60e-3], [10e-3, -10e-3, 0.0]]) / MU0
    fields[:, :, 1] = 2e-3 / MU0
    t_end, nt = 0.3e-9, 16
    t = np.linspace(0, t_end, nt)
    prob = MicromagProblem(res, L, solver="explicit", alpha=GAMMA * 1.0, gamma=0.0, tol=1e-6, nt_conv=nt - 1,
                           conv_tol=1e-3)
    prob.t_conv[:] = t[1:]
    t_out, M, _ = prob.run_batch(t_end, nt, fields, m0=m0.transpose(0, 2, 1))
    assert M.shape == (B, nt, n, K, 3)
    K32 = device_tensor(res, L)
    exits = 0
    for b in range(B):
        hext = np.zeros((K, 4))
        hext[:, 1:] = fields[b]
        P = oracle.Problem(res, L, solver=1, mode=2, gamma=0.0, alpha=GAMMA * 1.0, hext=hext, K32=K32)
        m = m0[b].reshape(-1)
        for k in range(K):
            P.set_hext_ind(k)
            to, yo, _, so = P.solve(t, m, tol=1e-6, t_conv=t[1:], conv_tol=1e-3)
            st = prob.last_stats[k][b]
            assert st["converged_at"] == so["converged_at"] and st["f_evals"] == so["f_evals"], (b, k, st, so)
            got = M[b, :, :, k, :].transpose(0, 2, 1).reshape(nt, -1)
            assert np.array_equal(got, yo), (b, k)
            kc = so["converged_at"]
            exits += kc >= 0
            m = yo[kc if kc >= 0 else nt - 1]
    assert exits >= 3
