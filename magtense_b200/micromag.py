"""Drop-in ``MicromagProblem`` for the micromagnetic path of MagTense.

Mirrors ``python/src/magtense/micromag.py`` of the reference (constructor
keywords and defaults :46-80, ``m0`` setter :152-168, option maps :174-211,
``run_simulation`` :213-268) and the Fortran behaviour behind it
(FortranToPythonIO.f90:429-489 -> SolveLandauLifshitzEquation,
LandauLifshitzEquationSolver.f90:50-209).  Everything is computed by the
sm_100a kernels of libmagtense_b200.so; there is no CPU path.

Differences from the reference, all deliberate:
  * ``cuda`` is accepted and ignored (the device path is the only path).
  * ``demag_approx`` "threshold" / "threshold_fraction" with ``dem_thres``
    run the thresholded-sparse demag of the reference; the FFT approximations,
    ``cvode=True`` and non-uniform grids raise NotImplementedError (not on this
    path).  After ``run_simulation`` the kept entries and the threshold used
    are in ``demag_sparse``.
  * ``H_exc, H_ext, H_dem, H_ani`` are computed when ``ReturnHall=1``
    (StoreHeffComponents :306-349); otherwise they are zeros (the reference
    leaves the flag uninitialised on its Python path).
  * explicit mode returns M with shape (nt, n, nt_Hext, 3), chaining m between
    field rows as the solver does (:165-186).
  * ``renormalize=True`` (keyword only, default False) rescales every cell's m
    to unit length after each accepted step.
  * explicit mode: after a convergence exit (t_conv / conv_tol) the next field
    starts from the sample the exit stored; the reference starts it from sample
    nt, which that run did not write.
"""
from __future__ import annotations

import os
from typing import List, Optional, Union

import numpy as np
import torch

from .solver import Solver, grid_points


class MicromagProblem:
    """Micromagnetic problem solved with the B200 kernels (same arguments as the reference)."""

    def __init__(
        self,
        res: List[int],
        grid_L: List[float] = [500e-9, 125e-9, 3e-9],
        grid_nnod: int = 0,
        grid_type: Optional[str] = "uniform",
        prob_mode: Optional[str] = "new",
        solver: Optional[str] = "dynamic",
        m0: Union[None, int, float, List, np.ndarray] = None,
        A0: float = 1.3e-11,
        Ms: float = 8e5,
        K0: float = 0.0,
        alpha: float = 0.02,
        gamma: float = 0.0,
        max_T0: float = 2.0,
        nt_conv: int = 1,
        conv_tol: float = 1e-4,
        tol: float = 1e-4,
        thres: float = 1e-6,
        setTimeDis: int = 10,
        dem_thres: float = 0.0,
        demag_approx: Optional[str] = None,
        CV: float = 0.0,
        ReturnHall: int = 0,
        exch_nval: int = 1,
        exch_nrow: int = 1,
        filename: str = "t",
        cuda: bool = False,
        cvode: bool = False,
        precision: bool = False,
        n_threads: int = 1,
        N_ave: List[int] = [1, 1, 1],
        t_alpha: np.ndarray = np.zeros(1),
        alpha_fct=lambda t: np.atleast_2d(t).T * 0,
        *,
        renormalize: bool = False,
    ) -> None:
        ntot = int(np.prod(res))
        self.ntot = ntot
        self.grid_nnod = grid_nnod
        self.nt_conv = nt_conv
        self.exch_nval = exch_nval
        self.exch_nrow = exch_nrow
        self.grid_n = np.array(res, dtype=np.int32, order="F")
        self.grid_L = np.array(grid_L, dtype=np.float64, order="F")
        self.grid_pts = np.zeros(shape=(ntot, 3), dtype=np.float64, order="F")
        self.u_ea = np.zeros(shape=(ntot, 3), dtype=np.float64, order="F")
        self.grid_type = grid_type
        self.prob_mode = prob_mode
        self.solver = solver
        self.m0 = m0
        self.A0 = A0
        self.Ms = Ms
        self.K0 = K0
        self.alpha_mm = alpha
        self.gamma = gamma
        self.max_T0 = max_T0
        self.t_conv = np.zeros(shape=(nt_conv), dtype=np.float64, order="F")
        self.conv_tol = np.array(np.repeat(conv_tol, nt_conv), dtype=np.float64, order="F")
        self.tol = tol
        self.thres = thres
        self.setTimeDis = setTimeDis
        self.dem_thres = dem_thres
        self.dem_appr = demag_approx
        self.CV = CV
        self.ReturnHall = ReturnHall
        self.nt_alpha = len(t_alpha)
        self.alphat = np.zeros(shape=(self.nt_alpha, 2), dtype=np.float64, order="F")
        self.alphat[:, 0] = t_alpha
        self.alphat[:, 1] = np.asarray(alpha_fct(t_alpha)).reshape(-1)[: self.nt_alpha] if self.nt_alpha else []
        self.N_load = len(filename)
        self.N_file_in = filename
        self.N_ret = len(filename)
        self.N_file_out = filename
        self.cuda = int(cuda)
        self.cvode = int(cvode)
        self.precision = int(precision)
        self.n_threads = n_threads
        self.N_ave = np.array(N_ave, dtype=np.int32, order="F")
        self.renormalize = bool(renormalize)
        self.last_stats = None
        self._solver_obj = None
        self.demag_sparse = None

    # --- properties with the reference's option maps ---------------------
    @property
    def m0(self):
        return self._m0

    @m0.setter
    def m0(self, val):
        self._m0 = np.zeros(shape=(self.ntot, 3), dtype=np.float64, order="F")
        if isinstance(val, type(None)):
            theta = np.pi * np.random.rand(self.ntot)
            phi = 2 * np.pi * np.random.rand(self.ntot)
            self._m0[:, 0] = np.sin(theta) * np.cos(phi)
            self._m0[:, 1] = np.sin(theta) * np.sin(phi)
            self._m0[:, 2] = np.cos(theta)
        elif isinstance(val, (int, float)):
            self._m0[:] = val
        else:
            assert np.asarray(val).shape == (self.ntot, 3)
            self._m0 = np.asarray(val, dtype=np.float64, order="F")

    @property
    def dem_appr(self):
        return self._dem_appr

    @dem_appr.setter
    def dem_appr(self, val=None):
        self._dem_appr = {None: 1, "threshold": 2, "fft_thres": 3, "threshold_fraction": 4,
                          "fft_threshold_fraction": 5}[val]

    @property
    def grid_type(self):
        return self._grid_type

    @grid_type.setter
    def grid_type(self, val=None):
        self._grid_type = {None: -1, "uniform": 1, "tetrahedron": 2, "unstructuredPrisms": 3}[val]

    @property
    def prob_mode(self):
        return self._prob_mode

    @prob_mode.setter
    def prob_mode(self, val=None):
        self._prob_mode = {None: -1, "new": 1, "old": 2}[val]

    @property
    def solver(self):
        return self._solver

    @solver.setter
    def solver(self, val=None):
        self._solver = {None: -1, "explicit": 1, "dynamic": 2, "implicit": 3}[val]

    # --- solve -----------------------------------------------------------
    def _check_supported(self):
        if self._grid_type != 1:
            raise NotImplementedError("only grid_type='uniform' is on the B200 path")
        if self._dem_appr in (3, 5):
            raise NotImplementedError("FFT demag approximations are not on the B200 path")
        if self.cvode:
            raise NotImplementedError("the CVODE integrator is not on the B200 path (RKSUITE 'M' only)")
        if self._solver not in (1, 2):
            raise NotImplementedError("solver must be 'explicit' or 'dynamic'")
        if self.CV > 0:
            raise NotImplementedError("demag-field noise (CV > 0) is not on the B200 path")
        if np.prod(self.N_ave) > 1:
            print("Averaging the N_tensor not supported for this tile type")

    def _make_solver(self):
        s = Solver(self.grid_n, self.grid_L, A0=self.A0, Ms=self.Ms, K0=self.K0, u_ea=self.u_ea)
        if self.N_load > 2:
            # loadDemagTensorFromDisk (MagTenseMicroMagPyIO.f90:251-271): 6 raw FP32 records
            s.load_tensor_colmajor(load_demag_tensor(self.N_file_in, self.ntot))
        else:
            s.assemble()
        if self._dem_appr in (2, 4):   # ApplyThresholdDense (DemagAuxFunctions.f90:20-122)
            self.demag_sparse = s.set_demag_threshold("threshold" if self._dem_appr == 2 else "threshold_fraction",
                                                      self.dem_thres)
        return s

    def run_simulation(self, t_end, nt, fct_h_ext, nt_h_ext):
        self._check_supported()
        t = np.linspace(0, t_end, nt)
        h_ext = np.zeros(shape=(nt_h_ext, 4), dtype=np.float64, order="F")
        h_ext[:, 0] = np.linspace(0, t_end, nt_h_ext)
        h_ext[:, 1:4] = fct_h_ext(np.linspace(0, t_end, nt_h_ext))
        n = self.ntot
        s = self._make_solver()
        self._solver_obj = s
        alpha_tab = np.ascontiguousarray(self.alphat)
        m0 = np.concatenate((self.m0[:, 0], self.m0[:, 1], self.m0[:, 2]), axis=None)
        n_fields = nt_h_ext if self._solver == 1 else 1
        M = np.zeros((nt, n, n_fields, 3))
        H = [np.zeros((nt, n, n_fields, 3)) for _ in range(4)] if self.ReturnHall == 1 else None
        t_out = np.zeros(nt)
        m_cur = torch.as_tensor(m0, device=s.device)
        stats = []
        for i in range(n_fields):
            s.set_dynamics(solver=self._solver, gamma=self.gamma, alpha=self.alpha_mm, alpha_tab=alpha_tab,
                           hext=np.ascontiguousarray(h_ext), hext_row=i, renormalize=self.renormalize)
            t_out, y, flags, st = s.integrate(t, m_cur, tol=self.tol, thres=self.thres, t_conv=self.t_conv,
                                              conv_tol=float(self.conv_tol[0]))
            stats.append(st)
            m_cur = y[_chain_sample(st, nt)].clone()
            yh = y.view(nt, 3, n).permute(0, 2, 1).cpu().numpy()
            M[:, :, i, :] = yh
            if H is not None:   # StoreHeffComponents: fields at the requested times
                for j in range(nt):
                    Hj, Hh, Hk, Hm = s.fields(t[j], y[j])
                    for arr, v in zip(H, (Hj, Hh, Hm, Hk)):
                        arr[j, :, i, :] = v.t().cpu().numpy()
        self.last_stats = stats if len(stats) > 1 else stats[0]
        pts = grid_points(self.grid_n, self.grid_L)
        if H is None:
            H = [np.zeros((nt, n, 1, 3)) for _ in range(4)]
        return t_out, M, pts, H[0], H[1], H[2], H[3]

    def run_batch(self, t_end, nt, h_ext, *, m0=None, alpha=None, precision="int8", keep_trajectory=True):
        """B instances of this problem in one call: one grid, material and demag
        tensor, and per instance its own applied field, damping, initial state and
        RKSUITE 'M' step control; every right-hand-side evaluation of all instances
        shares one demag GEMM (``BatchSolver``).  The reference solves one problem
        per call; its dataset workflow loops ``run_simulation`` over seeded fields
        (python/scripts/database.py:19-87).

        h_ext, dynamic solver: (B, nt_h_ext, 3) fields in A/m at the times
            linspace(0, t_end, nt_h_ext), or (B, 3) constant fields.
        h_ext, explicit solver: (B, 3), one quasi-static field per instance, or
            (B, K, 3), a branch of K fields per instance taken in turn, each from
            the state the previous one ended in (sample nt - 1, as
            LandauLifshitzEquationSolver.f90:165-186 chains its field rows), with
            the t_conv / conv_tol early exit of every field's run.
        m0: None (this problem's m0 for every instance) or (B, n, 3).
        alpha: None (this problem's alpha) or a scalar or (B,) array, as ``alpha``
            of the constructor; instances whose alpha is 0 follow this problem's
            alpha(t) table (``t_alpha``, ``alpha_fct``), as the reference's alpha().
        precision: "int8" (exact fixed-point product, the default), "fp32" (the
            reference's FP32 product), "bf16x3", "bf16x2" or "fp16s".
        Returns (t_out (B, nt), M (B, nt, n, K, 3) or None without the trajectory,
        pts (n, 3)), K = 1 except for an explicit branch; t_out is that of the last
        field; per-instance statistics go to ``self.last_stats`` (a list per
        field of a branch)."""
        from .solver import BatchSolver
        self._check_supported()
        if self.N_load > 2:
            raise NotImplementedError("run_batch assembles its tensor; loading one from disk is run_simulation only")
        if self._dem_appr != 1:
            raise NotImplementedError("run_batch runs the dense demag product; thresholded demag is run_simulation only")
        n = self.ntot
        h = np.asarray(h_ext, dtype=np.float64)
        if h.ndim not in (2, 3) or h.shape[-1] != 3:
            raise ValueError("h_ext must be (B, 3) or (B, K, 3)")
        branch = self._solver == 1 and h.ndim == 3
        if h.ndim == 2:
            h = np.repeat(h[:, None, :], 2, axis=1)
        B = h.shape[0]
        # one table per run: the dynamic solver's time table, or one quasi-static row per field
        rows = [h[:, k:k + 1, :] for k in range(h.shape[1])] if branch else [h]
        al = np.broadcast_to(np.asarray(self.alpha_mm if alpha is None else alpha, dtype=np.float64), (B,))
        if m0 is None:
            base = np.concatenate((self.m0[:, 0], self.m0[:, 1], self.m0[:, 2]))
            m0s = np.broadcast_to(base, (B, 3 * n)).copy()
        else:
            m0s = np.asarray(m0, dtype=np.float64).reshape(B, n, 3).transpose(0, 2, 1).reshape(B, 3 * n).copy()
        bs = BatchSolver(self.grid_n, self.grid_L, B, precision=precision, A0=self.A0, Ms=self.Ms, K0=self.K0,
                         u_ea=self.u_ea)
        M = None if not keep_trajectory else np.zeros((B, nt, n, len(rows), 3))
        stats = []
        try:
            bs.assemble()
            bs.tune()
            t = np.linspace(0, t_end, nt)
            m_cur = m0s
            for k, hk in enumerate(rows):
                ntab = hk.shape[1]
                tab = np.zeros((B, ntab, 4))
                tab[:, :, 0] = np.linspace(0, t_end, ntab)[None, :]
                tab[:, :, 1:] = hk
                bs.set_dynamics(hext=tab, alpha=al, solver=self._solver, gamma=self.gamma,
                                renormalize=self.renormalize,
                                alpha_tab=np.ascontiguousarray(self.alphat) if np.any(al == 0.0) else None)
                t_out, y, _, st = bs.integrate(t, m_cur, tol=self.tol, thres=self.thres, t_conv=self.t_conv,
                                               conv_tol=float(self.conv_tol[0]),
                                               keep_trajectory=keep_trajectory or k + 1 < len(rows))
                stats.append(st)
                if y is not None:
                    if M is not None:
                        M[:, :, :, k, :] = y.view(B, nt, 3, n).permute(0, 1, 3, 2).cpu().numpy()
                    m_cur = torch.stack([y[b, _chain_sample(st[b], nt)] for b in range(B)])
        finally:
            bs.close()
        self.last_stats = stats if branch else stats[0]
        return t_out, M, grid_points(self.grid_n, self.grid_L)


def _chain_sample(stats, nt):
    """The sample the next field of an explicit chain starts from: the last one
    (LandauLifshitzEquationSolver.f90:177 takes sample nt), or, after a
    convergence exit, the sample the exit stored.  The reference reads sample nt
    there too, which that run never wrote."""
    k = int(stats.get("converged_at", -1))
    return k if 0 <= k < nt else nt - 1


def load_demag_tensor(filename: str, n: int):
    """Read the reference's raw demag-tensor file: six records of n*n FP32, column-major
    (writeDemagTensorToDisk / loadDemagTensorFromDisk, MagTenseMicroMagPyIO.f90:221-271)."""
    raw = np.fromfile(filename, dtype=np.float32)
    if raw.size != 6 * n * n:
        raise ValueError(f"{filename}: expected 6*{n}*{n} float32 values, found {raw.size}")
    return [raw[k * n * n:(k + 1) * n * n].reshape((n, n), order="F") for k in range(6)]


def save_demag_tensor(filename: str, blocks) -> None:
    """Write six (n, n) blocks in the reference's raw record layout (column-major FP32)."""
    with open(filename, "wb") as f:
        for b in blocks:
            np.asarray(b, dtype=np.float32).ravel(order="F").tofile(f)
    os.chmod(filename, 0o644)
