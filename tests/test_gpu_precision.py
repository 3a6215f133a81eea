"""Precision study of the batched demag product (the precision configuration):
the 128x32x1 film of 4 nm x 4 nm x 3 nm cells (n = 4096), a batch of 512
quasi-static field steps (mu0 H along x swept from -100 to +100 mT, each tilted
in plane by a seeded 1 degree), demag product in FP32 (SIMT), split BF16
(bf16x3, bf16x2), row-scaled split FP16 (fp16s) and the exact int8 fixed-point
product, all against the FP64 oracle:

- H_d error: 256 seeded receiver rows of the FP64 tensor, for 16 of the 512
  instances, relative to the largest component;
- <m>(t) error: the same sweep on the 20x5x1 film, 0.05 ns at alpha_G = 1 from
  a shared seeded state, every output sample of 4 instances (all five
  precisions); and on the 128x32x1 film itself, all 512 instances over
  0.005 ns, both ends of the sweep against the FP64 oracle (all but bf16x2).

Bounds (the measured values are printed): H_d fp32 2e-5 (the reference's own
FP32 arithmetic), bf16x3 1e-4, bf16x2 1e-2, fp16s 1e-4 (small entries of a row
fall into the FP16 subnormal range), int8 1e-5; <m>(t) 1e-4 for all but bf16x2
(1e-2)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MU0 = 4 * np.pi * 1e-7
GAMMA = 2.211e5
PRECS = ["fp32", "bf16x3", "bf16x2", "fp16s", "int8"]
H_BOUND = {"fp32": 2e-5, "bf16x3": 1e-4, "bf16x2": 1e-2, "fp16s": 1e-4, "int8": 1e-5}
M_BOUND = {"fp32": 1e-4, "bf16x3": 1e-4, "bf16x2": 1e-2, "fp16s": 1e-4, "int8": 1e-4}


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    torch.cuda.set_device(0)
    return torch


def sweep_fields(B, seed):
    """mu0 H along x from -100 to +100 mT, each tilted in plane by a seeded 1 degree."""
    rng = np.random.default_rng(seed)
    mag = np.linspace(-100e-3, 100e-3, B) / MU0
    tilt = np.deg2rad(1.0) * rng.choice([-1.0, 1.0], B)
    return np.stack([mag * np.cos(tilt), mag * np.sin(tilt), np.zeros(B)], 1)


def shared_state(n, seed):
    rng = np.random.default_rng(seed)
    m = np.array([1.0, 0.2, 0.0])[:, None] + 0.1 * rng.standard_normal((3, n))
    return m / np.linalg.norm(m, axis=0)


def test_precision_demag_field_errors(torch_cuda, oracle):
    from magtense_b200 import BatchSolver
    res, L = [128, 32, 1], [512e-9, 128e-9, 3e-9]
    n, B = 4096, 512
    rng = np.random.default_rng(3)
    base = shared_state(n, 3)
    # per instance a different state: the shared state rotated in plane by a seeded angle
    ang = rng.uniform(-np.pi, np.pi, B)
    c, s = np.cos(ang)[:, None], np.sin(ang)[:, None]
    m = np.stack([c * base[0] - s * base[1], s * base[0] + c * base[1], np.broadcast_to(base[2], (B, n))], 1)
    rows = np.sort(rng.choice(n, 256, replace=False))
    _, K64 = oracle.assemble(res, L, rows=rows, fp32=False, fp64=True)
    check = np.linspace(0, B - 1, 16).astype(int)
    Href = np.stack([oracle.demag_rows(None, K64, m[b], 8e5, mode=1) for b in check])   # (16, 3, 256)
    errs = {}
    for prec in PRECS:
        bs = BatchSolver(res, L, B, precision=prec)
        bs.assemble()
        H = bs.demag_field(torch_cuda.as_tensor(m.reshape(B, -1), device="cuda")).cpu().numpy().reshape(B, 3, n)
        bs.close()
        errs[prec] = float(np.abs(H[check][:, :, rows] - Href).max() / np.abs(Href).max())
    print("\nH_d error vs FP64 (128x32x1, 512 instances):", {k: f"{v:.2e}" for k, v in errs.items()})
    for prec in PRECS:
        assert errs[prec] <= H_BOUND[prec], (prec, errs[prec])


def test_precision_mean_m_trajectory_errors(torch_cuda, oracle):
    from magtense_b200 import BatchSolver
    res, L = [20, 5, 1], [80e-9, 20e-9, 3e-9]
    n, B = 100, 16
    window = 0.05e-9
    Hf = sweep_fields(B, 5)
    hext = np.zeros((B, 2, 4))
    hext[:, 1, 0] = window
    hext[:, :, 1:] = Hf[:, None, :]
    m0 = np.broadcast_to(shared_state(n, 6), (B, 3, n)).copy()
    t = np.linspace(0, window, 26)
    check = [0, 5, 10, 15]
    ref = {}
    P64 = {b: oracle.Problem(res, L, mode=1, gamma=GAMMA, alpha=GAMMA * 1.0, hext=hext[b]) for b in check}
    for b in check:
        to, yo, _, _ = P64[b].solve(t, m0[b].reshape(-1), tol=1e-6)
        ref[b] = (to, yo.reshape(len(t), 3, n).mean(axis=2))
    errs, evals = {}, {}
    for prec in PRECS:
        bs = BatchSolver(res, L, B, precision=prec)
        bs.assemble()
        bs.set_dynamics(hext=hext, alpha=GAMMA * 1.0, gamma=GAMMA)
        t_out, y, _, st = bs.integrate(t, torch_cuda.as_tensor(m0.reshape(B, -1), device="cuda"), tol=1e-6)
        y = y.cpu().numpy().reshape(B, len(t), 3, n).mean(axis=3)
        bs.close()
        e, matched = 0.0, []
        for b in check:
            to, mref = ref[b]
            same = t_out[b] == to
            matched.append(float(same.mean()))
            # bf16x2's rounding noise drives the step size so far down that RKSUITE's
            # work limit displaces samples (flag 3): only the samples at equal times compare
            if prec != "bf16x2":
                assert same.mean() > 0.8, (prec, b)
            e = max(e, float(np.abs(y[b][same] - mref[same]).max()))
        errs[prec] = e
        if prec == "bf16x2":
            print("\nbf16x2 samples at the requested times:", matched)
        evals[prec] = int(np.median([s["f_evals"] for s in st]))
    print("\n<m>(t) error vs FP64 (20x5x1 sweep, alpha_G = 1):", {k: f"{v:.2e}" for k, v in errs.items()},
          "median RHS evaluations:", evals)
    for prec in PRECS:
        assert errs[prec] <= M_BOUND[prec], (prec, errs[prec])


def test_headline_geometry_mean_m_error_vs_fp64(torch_cuda, oracle):
    """The error statement of the batching configuration on its own geometry: the
    80x20x1 film from the s-state (seeded start relaxed 0.2 ns in zero field at
    alpha_G = 1), 4 instances of the seed-1000 in-plane field set, 0.1 ns at
    alpha_G = 0.02, tol 1e-6, output every 1 ps.  Both the int8 batched path and
    the plain FP32 path stay within 1e-4 of the FP64 oracle in <m>(t) (about 1e-7
    is measured over the full 1 ns)."""
    from magtense_b200 import BatchSolver, Solver
    res, L = [80, 20, 1], [500e-9, 125e-9, 3e-9]
    n, B = 1600, 4
    rng = np.random.default_rng(0)
    m = np.ones((3, n)) / np.sqrt(3) + 0.01 * rng.standard_normal((3, n))
    m = (m / np.linalg.norm(m, axis=0)).reshape(-1)
    s = Solver(res, L)
    s.assemble()
    s.set_dynamics(solver=2, gamma=GAMMA, alpha=GAMMA * 1.0, hext=np.array([[0, 0, 0, 0], [0.2e-9, 0, 0, 0.0]]))
    _, yr, _, _ = s.integrate(np.linspace(0, 0.2e-9, 3), torch_cuda.as_tensor(m, device="cuda"), tol=1e-6)
    m_s = yr[-1].cpu().numpy()
    r2 = np.random.default_rng(1000)
    ang = r2.uniform(0, 2 * np.pi, 256)
    mag = r2.uniform(0, 50e-3, 256) / MU0
    pick = [0, 85, 170, 255]
    Hf = np.stack([mag * np.cos(ang), mag * np.sin(ang), np.zeros(256)], 1)[pick]
    win = 0.1e-9
    t = np.linspace(0, win, 101)
    hext = np.zeros((B, 2, 4))
    hext[:, 1, 0] = win
    hext[:, :, 1:] = Hf[:, None, :]
    bs = BatchSolver(res, L, B, precision="int8")
    bs.assemble()
    bs.set_dynamics(hext=hext, alpha=GAMMA * 0.02, gamma=GAMMA)
    t_b, y_b, _, st_b = bs.integrate(t, np.tile(m_s, (B, 1)), tol=1e-6)
    y_b = y_b.cpu().numpy().reshape(B, len(t), 3, n).mean(axis=3)
    bs.close()
    _, K64 = oracle.assemble(res, L, fp32=False, fp64=True)
    worst = {"int8": 0.0, "fp32": 0.0}
    for b in range(B):
        s.set_dynamics(solver=2, gamma=GAMMA, alpha=GAMMA * 0.02, hext=hext[b])
        t_p, y_p, _, _ = s.integrate(t, torch_cuda.as_tensor(m_s, device="cuda"), tol=1e-6)
        y_p = y_p.cpu().numpy().reshape(len(t), 3, n).mean(axis=2)
        P = oracle.Problem(res, L, mode=1, gamma=GAMMA, alpha=GAMMA * 0.02, hext=hext[b], K64=K64)
        t_r, y_r, _, _ = P.solve(t, m_s, tol=1e-6)
        y_r = y_r.reshape(len(t), 3, n).mean(axis=2)
        for name, tg, yg in (("int8", t_b[b], y_b[b]), ("fp32", t_p, y_p)):
            same = tg == t_r
            assert same.mean() > 0.95
            worst[name] = max(worst[name], float(np.abs(yg[same] - y_r[same]).max()))
    print(f"80x20x1, 4 instances, 0.1 ns: max |<m> - <m>_FP64| {worst}")
    assert worst["int8"] <= 1e-4 and worst["fp32"] <= 1e-4, worst


def test_precision_config_geometry_mean_m_error(torch_cuda, oracle):
    """<m>(t) error on the precision configuration's own geometry: the 128x32x1 film
    (n = 4096), all 512 sweep instances relaxing at alpha_G = 1 from the shared state
    over 0.005 ns (output every 1 ps), each batched precision against the FP64 oracle
    at both ends of the sweep (-100 and +100 mT).  bf16x2 (1e-2 class) is covered on
    the 20x5x1 film above."""
    from magtense_b200 import BatchSolver
    res, L = [128, 32, 1], [512e-9, 128e-9, 3e-9]
    n, B = 4096, 512
    win = 0.005e-9
    Hf = sweep_fields(B, 5)
    m_sh = shared_state(n, 6).reshape(-1)
    hext = np.zeros((B, 2, 4))
    hext[:, 1, 0] = win
    hext[:, :, 1:] = Hf[:, None, :]
    t = np.linspace(0, win, 6)
    check = [0, B - 1]
    _, K64 = oracle.assemble(res, L, fp32=False, fp64=True)
    ref = {}
    for b in check:
        P = oracle.Problem(res, L, mode=1, gamma=GAMMA, alpha=GAMMA * 1.0, hext=hext[b], K64=K64)
        to, yo, _, _ = P.solve(t, m_sh, tol=1e-6)
        ref[b] = (to, yo.reshape(len(t), 3, n).mean(axis=2))
    del K64
    m0 = torch_cuda.as_tensor(np.tile(m_sh, (B, 1)), device="cuda")
    errs, matched = {}, {}
    for prec in ("fp32", "bf16x3", "fp16s", "int8"):
        bs = BatchSolver(res, L, B, precision=prec)
        bs.assemble()
        bs.set_dynamics(hext=hext, alpha=GAMMA * 1.0, gamma=GAMMA)
        t_out, y, _, _ = bs.integrate(t, m0, tol=1e-6)
        y = y.view(B, len(t), 3, n)[check].mean(dim=3).cpu().numpy()
        bs.close()
        e = 0.0
        for k, b in enumerate(check):
            to, mref = ref[b]
            same = t_out[b] == to
            matched[prec] = min(matched.get(prec, 1.0), float(same.mean()))
            # bf16x3's FP32-accumulated rounding noise drives the step size down on this
            # geometry (about 10^4 evaluations per instance against 600 for int8), so
            # RKSUITE's 5000-evaluation return displaces the later samples (flag 3): only
            # the samples at equal times compare
            assert same.mean() > (0.5 if prec == "bf16x3" else 0.8), (prec, b)
            e = max(e, float(np.abs(y[k][same] - mref[same]).max()))
        errs[prec] = e
    print("\n<m>(t) error vs FP64 (128x32x1, 512 instances, 0.005 ns, alpha_G = 1):",
          {k: f"{v:.2e}" for k, v in errs.items()}, "samples at the requested times:", matched)
    for prec, e in errs.items():
        assert e <= M_BOUND[prec], (prec, e)
