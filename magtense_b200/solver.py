"""Device-side solver object: one handle of libmagtense_b200.so plus torch-owned buffers.

PyTorch provides device memory and streams; all arithmetic runs in the
library's sm_100a kernels.  Vectors follow the reference layout
``[mx(0..n-1), my, mz]`` in FP64 (LandauLifshitzEquationSolver.f90:121,234-236).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import check

MU0 = 4 * np.pi * 1e-7


def _stream(stream=None):
    s = torch.cuda.current_stream() if stream is None else stream
    return C.c_void_p(s.cuda_stream)


def _dptr(t: torch.Tensor):
    return C.c_void_p(t.data_ptr())


def _np_d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def grid_points(res, grid_L) -> np.ndarray:
    """Cell centres (n, 3), x fastest (setupGrid, LandauLifshitzEquationSolver.f90:815-872)."""
    nx, ny, nz = (int(v) for v in res)
    axes = []
    for nn, L in zip((nx, ny, nz), grid_L):
        if nn > 1:
            d = L / nn
            axes.append(np.array([(-(L / 2.0) + i * d) + d / 2.0 for i in range(nn)]))
        else:
            axes.append(np.zeros(1))
    X = np.empty((nz, ny, nx, 3))
    X[..., 0] = axes[0][None, None, :]
    X[..., 1] = axes[1][None, :, None]
    X[..., 2] = axes[2][:, None, None]
    return X.reshape(nx * ny * nz, 3)


def shard_rows(n, rank, world):
    """Receiver cells [c0, c0 + nc) of row shard `rank` of `world` (as mt_set_row_shard)."""
    c0 = (n * rank) // world
    return c0, (n * (rank + 1)) // world - c0


class Solver:
    """Uniform-grid micromagnetic problem resident on one GPU.

    shard=(rank, world): this object is one row shard of the instance; it holds the
    tensor rows of its cells only (``shard_rows``), and only ``integrate`` runs it,
    at the same time as the other ranks' (see ``magtense_b200.shard.open_row_shard``
    for one process per GPU, ``link_shards_local`` and ``integrate_shards_local`` for
    all ranks on one device)."""

    def __init__(self, res, grid_L, *, A0=1.3e-11, Ms=8e5, K0=0.0, u_ea=None, device=None, shard=None):
        if not torch.cuda.is_available():
            raise RuntimeError("magtense_b200 needs a CUDA device (no CPU path exists)")
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        nx, ny, nz = (int(v) for v in res)
        self.res = (nx, ny, nz)
        self.grid_L = tuple(float(v) for v in grid_L)
        self.n = nx * ny * nz
        L = _lib.lib()
        g = _lib.Grid(nx, ny, nz, *self.grid_L)
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            check(L.mt_create(C.byref(g), C.byref(h)), "mt_create")
        self._h = h
        self.shard = None
        if shard is not None:
            rank, world = (int(v) for v in shard)
            check(L.mt_set_row_shard(self._h, rank, world), "mt_set_row_shard")
            self.shard = (rank, world)
        self.set_material(A0, Ms, K0, u_ea)
        self._have_tensor = False

    # ---------------------------------------------------------------- setup
    def set_material(self, A0, Ms, K0, u_ea=None):
        n = self.n
        self.A0 = float(A0)
        self.Ms = _np_d(np.broadcast_to(np.asarray(Ms, dtype=np.float64), (n,)))
        self.K0 = _np_d(np.broadcast_to(np.asarray(K0, dtype=np.float64), (n,)))
        self.u_ea = np.zeros((n, 3)) if u_ea is None else _np_d(np.asarray(u_ea, dtype=np.float64).reshape(n, 3))
        check(_lib.lib().mt_set_material(self._h, self.A0, self.Ms.ctypes.data_as(_lib.D),
                                         self.K0.ctypes.data_as(_lib.D), self.u_ea.ctypes.data_as(_lib.D)),
              "mt_set_material")

    def set_dynamics(self, *, solver=2, gamma=0.0, alpha=0.0, alpha_tab=None, hext=None, hext_row=0,
                     renormalize=False):
        at = np.zeros((1, 2)) if alpha_tab is None else _np_d(alpha_tab).reshape(-1, 2)
        he = np.zeros((2, 4)) if hext is None else _np_d(hext).reshape(-1, 4)
        self._tables = (at, he)
        check(_lib.lib().mt_set_dynamics(self._h, int(solver), float(gamma), float(alpha),
                                         at.ctypes.data_as(_lib.D), at.shape[0], he.ctypes.data_as(_lib.D),
                                         he.shape[0], int(hext_row), int(bool(renormalize))), "mt_set_dynamics")

    def assemble(self, stream=None):
        """FP64 analytical prism tensor of every cell pair, stored FP32 on the device."""
        with torch.cuda.device(self.device):
            check(_lib.lib().mt_assemble_demag(self._h, _stream(stream)), "mt_assemble_demag")
        self._have_tensor = True

    def load_tensor_colmajor(self, blocks):
        """Six (n, n) FP32 blocks Kxx Kxy Kxz Kyy Kyz Kzz, K[:, src] column-major as the reference."""
        bl = [np.asfortranarray(np.asarray(b, dtype=np.float32).reshape(self.n, self.n)) for b in blocks]
        ptrs = [b.ctypes.data_as(_lib.F) for b in bl]
        with torch.cuda.device(self.device):
            check(_lib.lib().mt_load_demag_colmajor(self._h, *ptrs), "mt_load_demag_colmajor")
        self._have_tensor = True

    def set_demag_threshold(self, approx, value, stream=None):
        """Thresholded-sparse demag: approx "threshold" keeps |K| > value, "threshold_fraction"
        removes the fraction value of the positive entries (the reference's bisection), None
        returns to the dense product.  Returns (kept entries, threshold used)."""
        code = {None: 1, "threshold": 2, "threshold_fraction": 4}[approx]
        nnz = C.c_longlong(0)
        thr = C.c_float(0.0)
        with torch.cuda.device(self.device):
            check(_lib.lib().mt_set_demag_threshold(self._h, code, float(value), C.byref(nnz), C.byref(thr),
                                                    _stream(stream)), "mt_set_demag_threshold")
        return nnz.value, thr.value

    def get_tensor_colmajor(self):
        """The six FP32 blocks as (n, n) arrays with K[i, j] = field at receiver i from source j."""
        out = [np.empty((self.n, self.n), dtype=np.float32, order="F") for _ in range(6)]
        with torch.cuda.device(self.device):
            check(_lib.lib().mt_get_demag_colmajor(self._h, *[o.ctypes.data_as(_lib.F) for o in out]),
                  "mt_get_demag_colmajor")
        return out

    # ---------------------------------------------------------------- fields
    def _vec(self, m):
        m = torch.as_tensor(m, dtype=torch.float64, device=self.device).reshape(3 * self.n)
        return m.contiguous()

    def demag_field(self, m, stream=None):
        """Internal demag field -Ms K m (FP32 product), shape (3, n)."""
        m = self._vec(m)
        out = torch.empty(3 * self.n, dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            check(_lib.lib().mt_demag_field(self._h, _dptr(m), _dptr(out), _stream(stream)), "mt_demag_field")
        return out.view(3, self.n)

    def fields(self, t, m, stream=None):
        """(H_exc, H_ext, H_ani, H_dem), each (3, n), the reference's internal sign."""
        m = self._vec(m)
        outs = [torch.empty(3 * self.n, dtype=torch.float64, device=self.device) for _ in range(4)]
        with torch.cuda.device(self.device):
            check(_lib.lib().mt_fields(self._h, float(t), _dptr(m), *[_dptr(o) for o in outs], _stream(stream)),
                  "mt_fields")
        return tuple(o.view(3, self.n) for o in outs)

    def rhs(self, t, m, stream=None):
        m = self._vec(m)
        out = torch.empty(3 * self.n, dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            check(_lib.lib().mt_rhs(self._h, float(t), _dptr(m), _dptr(out), _stream(stream)), "mt_rhs")
        return out

    def rhs_vjp(self, t, m, lam, stream=None):
        """Vector-Jacobian product of rhs at (t, m) for the cotangent lam (3n):
        returns (d/dm (3n), d/dhe (3n), d/dMs (n)); d/dhext = -(d/dhe).reshape(3, n).sum(1)."""
        m = self._vec(m)
        lam = self._vec(lam)
        gm = torch.empty(3 * self.n, dtype=torch.float64, device=self.device)
        ghe = torch.empty_like(gm)
        gms = torch.empty(self.n, dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            check(_lib.lib().mt_rhs_vjp(self._h, float(t), _dptr(m), _dptr(lam), _dptr(gm), _dptr(ghe), _dptr(gms),
                                        _stream(stream)), "mt_rhs_vjp")
        return gm, ghe, gms

    # ---------------------------------------------------------------- integrate
    def integrate(self, t, m0, *, tol=1e-4, thres=1e-6, t_conv=None, conv_tol=1e-4, y_out=None, stream=None):
        """MagTense_ODE_RKSuite on the device.

        Returns (t_out[nt] numpy, y_out (nt, 3n) cuda FP64, flags[nt] numpy, stats dict).
        """
        t = _np_d(t).reshape(-1)
        nt = t.shape[0]
        m0 = self._vec(m0)
        tc = np.zeros(1) if t_conv is None else _np_d(t_conv).reshape(-1)
        if y_out is None:
            y_out = torch.zeros((nt, 3 * self.n), dtype=torch.float64, device=self.device)
        t_out = np.zeros(nt)
        flags = np.zeros(nt, dtype=np.int32)
        st = _lib.Stats()
        with torch.cuda.device(self.device):
            rc = _lib.lib().mt_integrate(self._h, t.ctypes.data_as(_lib.D), nt, _dptr(m0), float(tol), float(thres),
                                         tc.ctypes.data_as(_lib.D), tc.shape[0], float(conv_tol),
                                         t_out.ctypes.data_as(_lib.D), _dptr(y_out), flags.ctypes.data_as(_lib.I),
                                         C.byref(st), _stream(stream))
        check(rc, "mt_integrate")
        return t_out, y_out, flags, st.as_dict()

    # ---------------------------------------------------------------- row shards
    @property
    def shard_cells(self):
        """(c0, nc): the receiver cells this shard owns (the whole grid without shards)."""
        return (0, self.n) if self.shard is None else shard_rows(self.n, *self.shard)

    def shard_region(self):
        """(device address, bytes) of this rank's exchange region, allocated on first use."""
        p = C.c_void_p()
        nb = C.c_size_t()
        with torch.cuda.device(self.device):
            check(_lib.lib().mt_shard_region(self._h, C.byref(p), C.byref(nb)), "mt_shard_region")
        return p.value, nb.value

    def shard_ipc_handle(self) -> bytes:
        """The CUDA IPC handle (64 bytes) of this rank's exchange region."""
        self.shard_region()
        buf = C.create_string_buffer(64)
        with torch.cuda.device(self.device):
            check(_lib.lib().mt_shard_ipc_handle(self._h, buf), "mt_shard_ipc_handle")
        return buf.raw

    def shard_open_peers(self, handles):
        """Map the other ranks' regions from their IPC handles (one per rank, rank order)."""
        blob = b"".join(bytes(hd) for hd in handles)
        if len(blob) != 64 * self.shard[1]:
            raise ValueError("need one 64-byte handle per rank")
        buf = C.create_string_buffer(blob, len(blob))
        with torch.cuda.device(self.device):
            check(_lib.lib().mt_shard_open_peers(self._h, buf), "mt_shard_open_peers")

    def shard_set_peers(self, regions):
        """The ranks' regions as device addresses valid in this process (rank order)."""
        arr = (C.c_void_p * len(regions))(*[int(r) for r in regions])
        check(_lib.lib().mt_shard_set_peers(self._h, arr), "mt_shard_set_peers")

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.lib().mt_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def integrate_ragged(solvers, t, m0s, *, tol=1e-4, thres=1e-6, graph=True, stream=None):
    """Integrate several independent single-instance problems (each its own ``Solver``:
    grid, tensor, material and dynamics set) over the same output times in one
    persistent launch, each on its own group of SMs with its own adaptive steps.

    m0s: one (3 n_k,) state per solver.  Returns (t_out (K, nt), [y_k (nt, 3 n_k)],
    flags (K, nt), stats list).  graph: replay the launch sequence from a CUDA graph."""
    K = len(solvers)
    t = _np_d(t).reshape(-1)
    nt = t.shape[0]
    dev = solvers[0].device
    m0t = [torch.as_tensor(m, dtype=torch.float64, device=dev).reshape(-1).contiguous() for m in m0s]
    ys = [torch.zeros((nt, 3 * sv.n), dtype=torch.float64, device=dev) for sv in solvers]
    hs = (VPA * K)(*[sv._h.value for sv in solvers])
    m0p = (VPA * K)(*[m.data_ptr() for m in m0t])
    yp = (VPA * K)(*[y.data_ptr() for y in ys])
    t_out = np.zeros((K, nt))
    flags = np.zeros((K, nt), dtype=np.int32)
    st = (_lib.Stats * K)()
    with torch.cuda.device(dev):
        rc = _lib.lib().mt_integrate_ragged(hs, K, t.ctypes.data_as(_lib.D), nt, m0p, float(tol), float(thres),
                                            t_out.ctypes.data_as(_lib.D), yp, flags.ctypes.data_as(_lib.I), st,
                                            1 if graph else 0, _stream(stream))
    check(rc, "mt_integrate_ragged")
    return t_out, ys, flags, [x.as_dict() for x in st]


def link_shards_local(shards):
    """Give every row shard of one instance on ONE device the other ranks' regions."""
    regions = [sv.shard_region()[0] for sv in shards]
    for sv in shards:
        sv.shard_set_peers(regions)


def integrate_shards_local(shards, t, m0, *, tol=1e-4, thres=1e-6, t_conv=None, conv_tol=1e-4, stream=None):
    """All row shards of one instance (``Solver(shard=(r, W))`` for r < W, linked with
    ``link_shards_local``) integrated on one device as CTA groups of one launch: the
    multi-GPU code path with its peer stores landing in local memory.  Returns what
    ``Solver.integrate`` returns, for the whole instance."""
    W = len(shards)
    sv0 = shards[0]
    t = _np_d(t).reshape(-1)
    nt = t.shape[0]
    m0 = sv0._vec(m0)
    tc = np.zeros(1) if t_conv is None else _np_d(t_conv).reshape(-1)
    y_out = torch.zeros((nt, 3 * sv0.n), dtype=torch.float64, device=sv0.device)
    t_out = np.zeros(nt)
    flags = np.zeros(nt, dtype=np.int32)
    st = _lib.Stats()
    hs = (VPA * W)(*[sv._h.value for sv in shards])
    with torch.cuda.device(sv0.device):
        rc = _lib.lib().mt_integrate_shards_local(hs, W, t.ctypes.data_as(_lib.D), nt, _dptr(m0), float(tol),
                                                  float(thres), tc.ctypes.data_as(_lib.D), tc.shape[0],
                                                  float(conv_tol), t_out.ctypes.data_as(_lib.D), _dptr(y_out),
                                                  flags.ctypes.data_as(_lib.I), C.byref(st), _stream(stream))
    check(rc, "mt_integrate_shards_local")
    return t_out, y_out, flags, st.as_dict()


VPA = C.c_void_p

PRECISIONS = {"fp32": 0, "bf16x3": 1, "bf16x2": 2, "fp16s": 3, "int8": 4}


class BatchSolver:
    """B instances sharing one uniform grid, material and demag tensor.

    Each instance has its own applied-field table, damping and initial state,
    and its own RKSUITE 'M' step control; all demag products of one
    right-hand-side evaluation form one GEMM.  ``precision``:

    - "fp32": FP32 SIMT, the reference's arithmetic;
    - "bf16x3" / "bf16x2": split-BF16 on the tcgen05 tensor cores, FP32 accumulate;
    - "fp16s": row-scaled split-FP16 on the tensor cores, FP32 accumulate;
    - "int8": exact fixed-point product on the integer tensor pipe (tensor rows
      as 24-bit fixed point, m as rint(m 2^30), twelve int8 limb products summed
      exactly).  It has no rounding noise, so the step-size control sees the
      dynamics instead of FP32 rounding; needs |m| < 1.96.
    """

    def __init__(self, res, grid_L, B, *, precision="bf16x3", A0=1.3e-11, Ms=8e5, K0=0.0, u_ea=None, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("magtense_b200 needs a CUDA device (no CPU path exists)")
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        nx, ny, nz = (int(v) for v in res)
        self.res = (nx, ny, nz)
        self.grid_L = tuple(float(v) for v in grid_L)
        self.n = nx * ny * nz
        self.B = int(B)
        self.precision = precision
        g = _lib.Grid(nx, ny, nz, *self.grid_L)
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            check(_lib.lib().mt_batch_create(C.byref(g), self.B, PRECISIONS[precision], C.byref(h)), "mt_batch_create")
        self._h = h
        n = self.n
        Ms_ = _np_d(np.broadcast_to(np.asarray(Ms, dtype=np.float64), (n,)))
        K0_ = _np_d(np.broadcast_to(np.asarray(K0, dtype=np.float64), (n,)))
        u = np.zeros((n, 3)) if u_ea is None else _np_d(np.asarray(u_ea, dtype=np.float64).reshape(n, 3))
        check(_lib.lib().mt_batch_set_material(self._h, float(A0), Ms_.ctypes.data_as(_lib.D),
                                               K0_.ctypes.data_as(_lib.D), u.ctypes.data_as(_lib.D)),
              "mt_batch_set_material")

    def assemble(self, stream=None):
        with torch.cuda.device(self.device):
            check(_lib.lib().mt_batch_assemble_demag(self._h, _stream(stream)), "mt_batch_assemble_demag")

    def set_dynamics(self, *, hext, alpha, solver=2, gamma=0.0, renormalize=False, alpha_tab=None):
        """hext: (B, nt_hext, 4) rows {t, Hx, Hy, Hz} per instance; alpha: scalar or (B,);
        alpha_tab: (nt_alpha, 2) rows {t, alpha}, the damping of the instances whose
        alpha is 0 (interpolated in t, 0 outside the table), as the reference's alpha()."""
        he = _np_d(hext).reshape(self.B, -1, 4)
        al = _np_d(np.broadcast_to(np.asarray(alpha, dtype=np.float64), (self.B,)))
        at = np.zeros((0, 2)) if alpha_tab is None else _np_d(alpha_tab).reshape(-1, 2)
        check(_lib.lib().mt_batch_set_alpha_table(self._h, at.ctypes.data_as(_lib.D), at.shape[0]),
              "mt_batch_set_alpha_table")
        self._tables = (he, al, at)
        check(_lib.lib().mt_batch_set_dynamics(self._h, int(solver), float(gamma), al.ctypes.data_as(_lib.D),
                                               he.ctypes.data_as(_lib.D), he.shape[1], int(bool(renormalize))),
              "mt_batch_set_dynamics")

    def tune(self, stream=None):
        """Autotune the int8 GEMM schedule (Stream-K CTA count and unit order per count of
        active 64-instance tiles) by timing the candidates on the device; the result is
        kept for this handle and cached for the process.  A no-op for other precisions."""
        with torch.cuda.device(self.device):
            check(_lib.lib().mt_batch_tune(self._h, _stream(stream)), "mt_batch_tune")
        return self.schedule()

    def schedule(self):
        """[(active tiles, Stream-K CTAs, "tile-major" | "row-major"), ...] in use."""
        cap = 2 * 64
        ctas = (C.c_int * cap)()
        order = (C.c_int * cap)()
        nt = C.c_int()
        check(_lib.lib().mt_batch_get_schedule(self._h, ctas, order, cap, C.byref(nt)), "mt_batch_get_schedule")
        return [(k + 1, int(ctas[k]), "row-major" if order[k] else "tile-major") for k in range(min(nt.value, cap))]

    def set_schedule(self, entries):
        """Set the schedule by hand: one (ctas, order 0|1) per active tile count 1..n_tiles."""
        n = len(entries)
        ctas = (C.c_int * n)(*[int(c) for c, _ in entries])
        order = (C.c_int * n)(*[int(o) for _, o in entries])
        check(_lib.lib().mt_batch_set_schedule(self._h, ctas, order, n), "mt_batch_set_schedule")

    def demag_field(self, m, stream=None):
        m = torch.as_tensor(m, dtype=torch.float64, device=self.device).reshape(self.B, 3 * self.n).contiguous()
        out = torch.empty_like(m)
        with torch.cuda.device(self.device):
            check(_lib.lib().mt_batch_demag_field(self._h, _dptr(m), _dptr(out), _stream(stream)),
                  "mt_batch_demag_field")
        return out.view(self.B, 3, self.n)

    def integrate(self, t, m0, *, tol=1e-4, thres=1e-6, t_conv=None, conv_tol=1e-4, keep_trajectory=True,
                  host_out=None, stream=None):
        """Returns (t_out (B, nt), y_out (B, nt, 3n) cuda FP64 or None, flags (B, nt), stats list).

        host_out: a pinned CPU FP64 tensor (B, nt, 3n) that receives the trajectories as
        the integration proceeds (finished samples after every relaunch, overlapped with
        the next); it is then returned in place of the device trajectories."""
        t = _np_d(t).reshape(-1)
        nt = t.shape[0]
        m0 = torch.as_tensor(m0, dtype=torch.float64, device=self.device).reshape(self.B, 3 * self.n).contiguous()
        tc = np.zeros(1) if t_conv is None else _np_d(t_conv).reshape(-1)
        y_out = torch.zeros((self.B, nt, 3 * self.n), dtype=torch.float64, device=self.device) \
            if keep_trajectory else None
        t_out = np.zeros((self.B, nt))
        flags = np.zeros((self.B, nt), dtype=np.int32)
        st = (_lib.Stats * self.B)()
        if host_out is not None:
            if not (host_out.is_pinned() and host_out.dtype == torch.float64 and host_out.is_contiguous()
                    and tuple(host_out.shape) == (self.B, nt, 3 * self.n)):
                raise ValueError("host_out must be a contiguous pinned float64 tensor of shape (B, nt, 3n)")
            if y_out is None:
                y_out = torch.zeros((self.B, nt, 3 * self.n), dtype=torch.float64, device=self.device)
            with torch.cuda.device(self.device):
                rc = _lib.lib().mt_batch_integrate_host(
                    self._h, t.ctypes.data_as(_lib.D), nt, _dptr(m0), float(tol), float(thres),
                    tc.ctypes.data_as(_lib.D), tc.shape[0], float(conv_tol), t_out.ctypes.data_as(_lib.D),
                    _dptr(y_out), C.c_void_p(host_out.data_ptr()), flags.ctypes.data_as(_lib.I), st,
                    _stream(stream))
            check(rc, "mt_batch_integrate_host")
            return t_out, host_out, flags, [x.as_dict() for x in st]
        with torch.cuda.device(self.device):
            rc = _lib.lib().mt_batch_integrate(self._h, t.ctypes.data_as(_lib.D), nt, _dptr(m0), float(tol),
                                               float(thres), tc.ctypes.data_as(_lib.D), tc.shape[0], float(conv_tol),
                                               t_out.ctypes.data_as(_lib.D),
                                               C.c_void_p(0) if y_out is None else _dptr(y_out),
                                               flags.ctypes.data_as(_lib.I), st, _stream(stream))
        check(rc, "mt_batch_integrate")
        return t_out, y_out, flags, [x.as_dict() for x in st]

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.lib().mt_batch_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
