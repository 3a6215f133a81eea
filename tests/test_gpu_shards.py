"""Row shards of one instance (mt_set_row_shard, mt_integrate_shards_local).

All ranks run on one device as CTA groups of one cooperative launch, the
multi-GPU code path with its peer stores landing in local memory.  When every
CTA owns the same cells as in the whole-instance run (n divisible by 8 * world,
below the SM cap) the demag sums, norms and steps are the same operations in the
same order, so the trajectory must equal mt_integrate's bit for bit; otherwise
it must agree within 1e-5 in m (FP32 product, different cell partition).  A
rank whose peers never arrive must give up with MT_ERR_TIMEOUT (bounded wait on
a flag that nothing sets), and its handle must then refuse to run."""
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


def film(nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    res, L = (nx, ny, nz), (nx * 6.25e-9, ny * 6.25e-9, nz * 3e-9)
    ang, mag = rng.uniform(0, 2 * np.pi), rng.uniform(5e-3, 50e-3) / MU0
    h = np.array([mag * np.cos(ang), mag * np.sin(ang), 0.0])
    m = np.ones((3, n)) / np.sqrt(3) + 0.05 * rng.standard_normal((3, n))
    m0 = (m / np.linalg.norm(m, axis=0)).reshape(-1)
    dyn = dict(solver=2, gamma=GAMMA, alpha=GAMMA * 0.05, hext=np.array([[0.0, *h], [1e-9, *h]]))
    return res, L, dyn, m0


def whole(res, L, dyn, renorm=False):
    from magtense_b200 import Solver
    s = Solver(res, L)
    s.set_dynamics(**dyn, renormalize=renorm)
    s.assemble()
    return s


def shards(res, L, dyn, world, renorm=False):
    from magtense_b200 import Solver, link_shards_local
    out = []
    for r in range(world):
        s = Solver(res, L, shard=(r, world))
        s.set_dynamics(**dyn, renormalize=renorm)
        s.assemble()
        out.append(s)
    link_shards_local(out)
    return out


T = np.linspace(0.0, 0.05e-9, 11)


@pytest.mark.parametrize("world", [2, 4, 8])
def test_shards_equal_whole_instance_bitwise(torch_cuda, world):
    from magtense_b200 import integrate_shards_local
    torch = torch_cuda
    res, L, dyn, m0 = film(40, 16, 1, 5)        # n = 640: 8 cells per CTA in both runs
    t1, y1, f1, s1 = whole(res, L, dyn).integrate(T, m0, tol=1e-6)
    sh = shards(res, L, dyn, world)
    t2, y2, f2, s2 = integrate_shards_local(sh, T, m0, tol=1e-6)
    assert np.array_equal(t1, t2)
    assert np.array_equal(f1, f2)
    assert s1["f_evals"] == s2["f_evals"] and s1["steps"] == s2["steps"], (s1, s2)
    assert torch.equal(y1, y2)
    # a second run on the same shards continues the barrier epochs and repeats the result
    t3, y3, _, s3 = integrate_shards_local(sh, T, m0, tol=1e-6)
    assert np.array_equal(t2, t3) and torch.equal(y2, y3) and s3["f_evals"] == s2["f_evals"]


def test_shards_renormalise_and_converge_bitwise(torch_cuda):
    from magtense_b200 import integrate_shards_local
    torch = torch_cuda
    res, L, dyn, m0 = film(40, 16, 1, 6)
    tc = np.linspace(0.0, 0.05e-9, 6)[1:]
    a = whole(res, L, dyn, renorm=True).integrate(T, m0, tol=1e-6, t_conv=tc, conv_tol=1e-3)
    b = integrate_shards_local(shards(res, L, dyn, 4, renorm=True), T, m0, tol=1e-6, t_conv=tc, conv_tol=1e-3)
    assert a[3]["converged_at"] == b[3]["converged_at"]
    assert np.array_equal(a[0], b[0])
    assert torch.equal(a[1], b[1])


def test_uneven_shards_across_z_planes(torch_cuda):
    """n = 814 over 3 ranks (271, 271, 272 cells); nz = 2, so the exchange stencil
    of every rank reads the other z-plane from other ranks' rows."""
    from magtense_b200 import integrate_shards_local
    torch = torch_cuda
    res, L, dyn, m0 = film(37, 11, 2, 7)
    t1, y1, _, s1 = whole(res, L, dyn).integrate(T, m0, tol=1e-6)
    t2, y2, _, s2 = integrate_shards_local(shards(res, L, dyn, 3), T, m0, tol=1e-6)
    assert s2["status"] == 0 and s2["n_out"] == len(T)
    k = min(s1["n_out"], s2["n_out"])
    same = t1[:k] == t2[:k]
    assert same.mean() > 0.9
    err = float((y1[:k][torch.as_tensor(same, device=y1.device)] - y2[:k][torch.as_tensor(same, device=y1.device)]).abs().max())
    assert err < 1e-5, err


def test_shard_handle_serves_only_integrate(torch_cuda):
    from magtense_b200 import MTError, Solver
    res, L, dyn, m0 = film(16, 4, 1, 8)
    s = Solver(res, L, shard=(1, 2))
    s.set_dynamics(**dyn)
    s.assemble()
    assert s.shard_cells == (32, 32)
    with pytest.raises(MTError):
        s.rhs(0.0, m0)
    with pytest.raises(MTError):
        s.demag_field(m0)
    with pytest.raises(MTError):            # peers not set yet
        s.integrate(T, m0)
    from magtense_b200 import _lib
    w = whole(res, L, dyn)
    assert _lib.lib().mt_set_row_shard(w._h, 0, 2) == -4     # MT_ERR_STATE: tensor already assembled
    assert _lib.lib().mt_set_row_shard(w._h, 2, 2) == -1     # MT_ERR_ARG


def test_rank_without_peers_times_out(torch_cuda, monkeypatch):
    """Rank 0 of 2 runs alone: its wait for rank 1's barrier flag runs out (1 s),
    the kernel returns, the host reads MT_ERR_TIMEOUT, and the handle refuses
    further runs.  Rank 1's region is real memory that no kernel writes."""
    from magtense_b200 import MTError
    monkeypatch.setenv("MAGTENSE_B200_SHARD_TIMEOUT_S", "1")
    res, L, dyn, m0 = film(16, 4, 1, 9)
    sh = shards(res, L, dyn, 2)
    with pytest.raises(MTError, match="cross-rank"):
        sh[0].integrate(T, m0)
    with pytest.raises(MTError, match="gave up"):
        sh[0].integrate(T, m0)
