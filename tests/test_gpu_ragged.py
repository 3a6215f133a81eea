"""Ragged batch (mt_integrate_ragged): films of different sizes (nx x nx/4 x 1
cells of 6.25 x 6.25 x 3 nm), each with its own tensor, field and adaptive
steps, in one persistent launch on per-instance CTA groups.  Each instance
must match the single-instance integrator (mt_integrate) on the same problem
within 1e-5 in m at the output times both reached (same FP32 arithmetic,
different cell partition); the CUDA-graph replay must match the plain
launches bit for bit."""
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


def films(nxs, seed):
    from magtense_b200 import Solver
    rng = np.random.default_rng(seed)
    out = []
    for nx in nxs:
        ny = max(1, nx // 4)
        res, L = (nx, ny, 1), (nx * 6.25e-9, ny * 6.25e-9, 3e-9)
        n = nx * ny
        s = Solver(res, L)
        s.assemble()
        ang, mag = rng.uniform(0, 2 * np.pi), rng.uniform(5e-3, 50e-3) / MU0
        h = np.array([mag * np.cos(ang), mag * np.sin(ang), 0.0])
        s.set_dynamics(solver=2, gamma=GAMMA, alpha=GAMMA * 0.05, hext=np.array([[0.0, *h], [1e-9, *h]]))
        m = np.ones((3, n)) / np.sqrt(3) + 0.05 * rng.standard_normal((3, n))
        out.append((s, (m / np.linalg.norm(m, axis=0)).reshape(-1)))
    return out


def test_ragged_matches_single_instance(torch_cuda):
    from magtense_b200 import integrate_ragged
    torch = torch_cuda
    probs = films([20, 48, 32, 60, 24], 3)
    t = np.linspace(0, 0.02e-9, 11)
    t_out, ys, flags, st = integrate_ragged([p[0] for p in probs], t, [p[1] for p in probs], tol=1e-6, graph=False)
    t_out_g, ys_g, _, st_g = integrate_ragged([p[0] for p in probs], t, [p[1] for p in probs], tol=1e-6, graph=True)
    for k, (s, m0) in enumerate(probs):
        assert np.array_equal(t_out[k], t_out_g[k])
        assert torch.equal(ys[k], ys_g[k]), k
        to, y1, fl, s1 = s.integrate(t, torch.as_tensor(m0, device="cuda"), tol=1e-6)
        same = t_out[k] == to
        assert same.mean() > 0.9, (k, st[k], s1)
        err = float((ys[k][torch.as_tensor(same, device="cuda")] - y1[torch.as_tensor(same, device="cuda")]).abs().max())
        assert err < 1e-5, (k, err)
        assert st[k]["status"] == 0
    assert st[0]["launches"] >= 1


def test_ragged_rejects_more_instances_than_sms(torch_cuda):
    from magtense_b200 import integrate_ragged
    from magtense_b200._lib import MTError
    torch = torch_cuda
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    probs = films([8], 5)
    s, m0 = probs[0]
    with pytest.raises(MTError):
        integrate_ragged([s] * (sms + 1), np.linspace(0, 1e-12, 2), [m0] * (sms + 1), tol=1e-4)


def test_ragged_regroups_finished_instances(torch_cuda, monkeypatch):
    """Short launches (MT_RAGGED_LAUNCH_S) make the small films finish while the large
    ones still run; their CTAs then join the unfinished groups.  Every instance still
    matches mt_integrate within 1e-5, and the graph replay the plain launches bit for bit."""
    from magtense_b200 import integrate_ragged
    torch = torch_cuda
    monkeypatch.setenv("MT_RAGGED_LAUNCH_S", "0.0005")
    probs = films([16, 96, 20, 80, 24], 5)
    t = np.linspace(0, 0.02e-9, 11)
    t_out, ys, _, st = integrate_ragged([p[0] for p in probs], t, [p[1] for p in probs], tol=1e-6, graph=False)
    t_out_g, ys_g, _, st_g = integrate_ragged([p[0] for p in probs], t, [p[1] for p in probs], tol=1e-6, graph=True)
    assert st[0]["launches"] > 3
    for k, (s, m0) in enumerate(probs):
        assert np.array_equal(t_out[k], t_out_g[k])
        assert torch.equal(ys[k], ys_g[k]), k
        to, y1, _, s1 = s.integrate(t, torch.as_tensor(m0, device="cuda"), tol=1e-6)
        same = t_out[k] == to
        assert same.mean() > 0.9, (k, st[k], s1)
        err = float((ys[k][torch.as_tensor(same, device="cuda")] - y1[torch.as_tensor(same, device="cuda")]).abs().max())
        assert err < 1e-5, (k, err)
        assert st[k]["status"] == 0
