"""muMAG standard problem 4 against the reference's own published-solution band.

The reference ships the mean and spread of the published muMAG solutions of
standard problem 4 (Published_solutions_field{1,2}.mat, committed here as
tests/golden/mumag_std4_published.npz by make_mumag_std4_fixture.py) and runs
the problem with its std_problem_4 workflow (python/examples/micromagnetism/
std_problem_4.py: relax m0 = 1/sqrt(3) at alpha = 4.42e3 with no precession
for 100 ns, then 1 ns at gamma = 2.21e5 in field 1 (-24.6, 4.3, 0) mT or field 2
(-35.5, -6.3, 0) mT; tol 1e-4).  Its own distance to the band is the integral
over the ns of |<m_j>(t) - mean_j(t)| summed over j
(Benchmark_using_mumag_std_problem_4/Benchmark_results.m:73-77); that is the
metric here, in ns.

These tests run that workflow through the drop-in surface (MicromagProblem:
plain FP32 path, and run_batch with the int8 tensor-core product), with the
outputs requested at the band's 1000 times, and check:
  * the distance to the band at the reference's 80x20x1 resolution;
  * that refining the grid moves the trajectory toward the band, so what
    remains at 80x20x1 is discretisation, not the solver;
  * that the device trajectory equals the CPU oracle's run of the same
    recipe (RKSUITE decisions, RHS and output times), within 1e-3 in <m>.
"""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MU0 = 4 * np.pi * 1e-7
GOLDEN = Path(__file__).resolve().parent / "golden" / "mumag_std4_published.npz"
FIELDS = {1: np.array([-24.6, 4.3, 0.0]), 2: np.array([-35.5, -6.3, 0.0])}
GRID_L = [500e-9, 125e-9, 3e-9]
ALPHA, GAMMA = 4.42e3, 2.21e5

# Band distance (ns) allowed for field 1 at 80x20x1: the measured distance is
# 0.095; a wrong sign, factor or missing term in the right-hand side moves the
# switching and puts the distance near or above 0.5.
BAND_BOUND_80x20 = 0.15


def published(field):
    z = np.load(GOLDEN)
    return z["t_ns"], z[f"field{field}_mean"], z[f"field{field}_err"]


def band_distance(mavg, field, t_out):
    """Benchmark_results.m:73-77: the published mean interpolated to the times the run
    returned (t_out, s), then sum_j trapz(t, |<m_j> - mean_j|) with t in ns.  A flag-3
    return every 5000 evaluations moves a sample to the internal time
    (RKSuitef90.f90:1374-1387), hence the interpolation, as the reference does."""
    t, mean, _ = published(field)
    tn = np.asarray(t_out) * 1e9
    return float(sum(np.trapezoid(np.abs(mavg[:, j] - np.interp(tn, t, mean[:, j])), tn) for j in range(3)))


def relax_hfct(t):
    return np.expand_dims(np.where(t < 1e-09, 1e-09 - t, 0), axis=1) * (np.array([1, 1, 1]) / MU0)


def s_state(res):
    from magtense_b200 import MicromagProblem
    p = MicromagProblem(res, GRID_L, m0=1 / np.sqrt(3), alpha=ALPHA)
    _, M, _, _, _, _, _ = p.run_simulation(100e-9, 200, relax_hfct, 2000)
    return np.squeeze(M, axis=2)[-1], p.last_stats


def dynamic_plain(res, m_s, field, tol=1e-4):
    from magtense_b200 import MicromagProblem
    p = MicromagProblem(res, GRID_L, m0=m_s, alpha=ALPHA, gamma=GAMMA, tol=tol)
    h = FIELDS[field] / 1000 / MU0
    t, M, _, _, _, _, _ = p.run_simulation(1e-9, 1000, lambda tt: np.expand_dims(tt > -1, axis=1) * h, 2000)
    return t, np.squeeze(M, axis=2).mean(axis=1), p.last_stats


@pytest.fixture(scope="module")
def film80():
    import torch
    torch.cuda.set_device(0)
    res = [80, 20, 1]
    m_s, st_relax = s_state(res)
    runs = {f: dynamic_plain(res, m_s, f) for f in (1, 2)}
    return res, m_s, st_relax, runs


@pytest.fixture(scope="module")
def film160(film80):
    res = [160, 40, 1]
    m_s, _ = s_state(res)
    return {f: dynamic_plain(res, m_s, f) for f in (1, 2)}


def test_plain_fp32_lies_near_the_published_band(film80):
    field = 1
    res, m_s, _, runs = film80
    t, mavg, st = runs[field]
    tp, mean, err = published(field)
    same = np.abs(t * 1e9 - tp) < 1e-9
    assert same.mean() > 0.99       # all samples at the band's times but the flag-3 ones
    d = band_distance(mavg, field, t)
    print(f"field {field}: band distance {d:.4f} ns, max |<m> - mean| {np.abs(mavg - mean)[same].max(axis=0)}, "
          f"evaluations {st['f_evals']}")
    assert np.all(np.abs(np.linalg.norm(mavg, axis=1)) <= 1.0 + 1e-9)
    assert d <= BAND_BOUND_80x20, d
    # the start and the first switching phase (first 0.1 ns) sit close to the published mean
    assert np.abs(mavg[:100] - mean[:100]).max() < 0.05


@pytest.mark.parametrize("field", [1, 2])
def test_refinement_moves_toward_the_band(film80, film160, field):
    """Halving the cell size (160x40x1, 3.125 nm cells, below the exchange length of
    about 5.7 nm) brings the trajectory onto the band: for field 1 the distance
    falls from about 0.095 to about 0.006 ns, so what remains at 80x20x1 is
    discretisation.  Field 2 switches through a different path at 80x20x1
    (distance about 0.26) and comes onto the band at 160x40x1 too (about 0.015)."""
    _, _, _, runs = film80
    d80 = band_distance(runs[field][1], field, runs[field][0])
    t2, mavg2, st2 = film160[field]
    d160 = band_distance(mavg2, field, t2)
    print(f"field {field}: band distance 80x20x1 {d80:.4f} ns, 160x40x1 {d160:.4f} ns ({st2['f_evals']} evaluations)")
    assert d160 < 0.25 * d80
    assert d160 < 0.03


def test_int8_batch_matches_plain_and_band(film80):
    """Both fields as two instances of one batched run with the exact int8 product.
    At the workflow's tol 1e-4 two runs whose products round differently take
    different steps, and over the switching their <m> part by a few 1e-3 (the
    integration error that tolerance allows); both sit at the same band distance."""
    from magtense_b200 import MicromagProblem
    res, m_s, _, runs = film80
    p = MicromagProblem(res, GRID_L, m0=m_s, alpha=ALPHA, gamma=GAMMA)
    h = np.stack([FIELDS[1], FIELDS[2]]) / 1000 / MU0
    t_out, M, _ = p.run_batch(1e-9, 1000, h, m0=np.stack([m_s, m_s]), precision="int8")
    for k, field in enumerate((1, 2)):
        mavg = M[k, :, :, 0, :].mean(axis=1)
        d = band_distance(mavg, field, t_out[k])
        d_plain = band_distance(runs[field][1], field, runs[field][0])
        same = t_out[k] == runs[field][0]
        diff = np.abs(mavg - runs[field][1])[same].max()
        print(f"int8 field {field}: band distance {d:.4f} ns (fp32 {d_plain:.4f}), max |<m>_int8 - <m>_fp32| "
              f"{diff:.2e}")
        if field == 1:
            assert d <= BAND_BOUND_80x20, d
        assert abs(d - d_plain) < 0.01
        assert diff < 2e-2, diff


def test_device_run_equals_oracle_run(film80, oracle):
    """The same recipe on the CPU oracle (the reference's FP32 product).  The relaxed
    states agree to 1e-4 (relaxation converges whatever the step sequence).  The
    dynamic part runs at tol 1e-6, where the integration error is small enough that
    the device and oracle trajectories, whose FP32 products sum in different orders,
    agree to 1e-3 in <m> over the whole ns."""
    res, m_s, st_relax, runs = film80
    n = int(np.prod(res))
    tt = np.linspace(0, 100e-9, 2000)
    hext = np.zeros((2000, 4))
    hext[:, 0] = tt
    hext[:, 1:] = relax_hfct(tt)
    P = oracle.Problem(res, GRID_L, mode=0, gamma=0.0, alpha=ALPHA, hext=hext)
    m0 = np.ones(3 * n) / np.sqrt(3)
    _, yo, _, so = P.solve(np.linspace(0, 100e-9, 200), m0, tol=1e-4)
    ms_o = yo[-1].reshape(3, n).T
    relax_diff = np.abs(ms_o - m_s).max()
    print(f"relaxed state: max |m_device - m_oracle| {relax_diff:.2e}; evaluations {st_relax['f_evals']} "
          f"(oracle {so['f_evals']})")
    assert relax_diff < 1e-4
    field = 1
    t_d, m_d, st_d = dynamic_plain(res, m_s, field, tol=1e-6)
    t1 = np.linspace(0, 1e-9, 2000)
    hd = np.zeros((2000, 4))
    hd[:, 0] = t1
    hd[:, 1:] = FIELDS[field] / 1000 / MU0
    P2 = oracle.Problem(res, GRID_L, mode=0, gamma=GAMMA, alpha=ALPHA, hext=hd, K32=P.K32)
    t_o, y2, _, s2 = P2.solve(np.linspace(0, 1e-9, 1000), yo[-1], tol=1e-6)
    mo = y2.reshape(1000, 3, n).mean(axis=2)
    same = t_o == t_d
    diff = np.abs(mo - m_d)[same].max()
    print(f"field {field}, tol 1e-6: max |<m>_device - <m>_oracle| {diff:.2e} over {same.sum()} samples; "
          f"evaluations {st_d['f_evals']} (oracle {s2['f_evals']}); band distance {band_distance(m_d, field, t_d):.4f} "
          f"(oracle {band_distance(mo, field, t_o):.4f}) ns")
    assert same.mean() > 0.99
    assert diff < 1e-3, diff
