"""Std-problem-4 dataset driver: every sequence of a database in one batched run.

Mirrors the reference's dataset workflow (python/scripts/database.py
``db_std_prob_4`` :19-87 with ``gen_s_state`` / ``gen_seq`` of
python/scripts/db_utils.py :14-82): a relaxed s-state, then per sequence a
seeded in-plane field (magnitude U[h_ext_n] mT, angle U[h_ext_a] degrees, the
same draws from ``numpy.random.default_rng(seed)``) applied from the s-state
for ``t_steps`` outputs ``t_per_step`` apart, at alpha = 4.42e3 and
gamma = 2.211e5.  The reference integrates the sequences one process call
after another; here they are the instances of one ``MicromagProblem.run_batch``
call.  Output layout as the reference's database: ``sequence``
(n, t_steps, 3, res_x, res_y) FP32 and ``field`` (n, 3) FP32 in mT.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

MU0 = 4 * np.pi * 1e-7
ALPHA = 4.42e3
GAMMA = 2.211e5


def std_prob_4_fields(n_seq, h_ext_a=(0, 360), h_ext_n=(0, 50), seed=0, intv=None):
    """(n, 3) applied fields in mT of the sequences of interval ``intv`` (all
    ``n_seq`` by default), drawn as the reference draws them (database.py:62-70).
    The reference fills an interval [lo, hi) from rows 0 .. hi - lo - 1 of its
    seeded draw table, whatever lo is, so an interval database with lo > 0
    repeats the fields of the first hi - lo sequences; this function returns
    the same rows."""
    rng = np.random.default_rng(seed)
    rnd = rng.random(size=(n_seq, 2))
    lo, hi = (0, n_seq) if intv is None else intv
    d = (h_ext_n[1] - h_ext_n[0]) * rnd[:, 0] + h_ext_n[0]
    theta = np.deg2rad((h_ext_a[1] - h_ext_a[0]) * rnd[:, 1] + h_ext_a[0])
    f = np.zeros((n_seq, 3))
    f[:, 0] = d * np.cos(theta)
    f[:, 1] = d * np.sin(theta)
    return f[: hi - lo]


def sequence_layout(M, res):
    """(t, n, 3) magnetisation, x fastest, to the database's (t, 3, res_x, res_y)
    (database.py:82-85)."""
    t = M.shape[0]
    return np.moveaxis(np.asarray(M).reshape(t, res[1], res[0], 3).swapaxes(1, 2), -1, 1)


def s_state(res, grid_size=(500e-9, 500e-9, 3e-9), t_end=100e-9, nt=200, nt_h_ext=2000):
    """The relaxed s-state (n, 3) of gen_s_state (db_utils.py:14-48): m0 = 1/sqrt(3)
    everywhere, a field along (1, 1, 1)/mu0 A/m that ramps down to zero over the
    first ns, alpha = 4.42e3, no precession, 100 ns."""
    from .micromag import MicromagProblem
    prob = MicromagProblem(res=list(res) + [1] if len(res) == 2 else list(res), grid_L=list(grid_size),
                           m0=1 / np.sqrt(3), alpha=ALPHA)
    h = np.array([1.0, 1.0, 1.0]) / MU0
    fct = lambda t: np.expand_dims(np.where(t < 1e-9, 1e-9 - t, 0), axis=1) * h   # noqa: E731
    _, M, _, _, _, _, _ = prob.run_simulation(t_end, nt, fct, nt_h_ext)
    return np.squeeze(M, axis=2)[-1]


def std_prob_4_sequences(m0_state, res, fields_mT, grid_size=(500e-9, 500e-9, 3e-9), t_steps=500,
                         t_per_step=4e-12, precision="int8"):
    """(n, t_steps, 3, res_x, res_y) FP32: every field of ``fields_mT`` (n, 3)
    applied from ``m0_state`` (n_cells, 3) as gen_seq does (db_utils.py:51-82),
    all sequences in one batched run.  Returns (sequences, per-sequence stats)."""
    from .micromag import MicromagProblem
    fields = np.asarray(fields_mT, dtype=np.float64).reshape(-1, 3)
    B = fields.shape[0]
    r3 = list(res) + [1] if len(res) == 2 else list(res)
    prob = MicromagProblem(res=r3, grid_L=list(grid_size), m0=np.asarray(m0_state, dtype=np.float64),
                           alpha=ALPHA, gamma=GAMMA)
    h = fields / 1000 / MU0
    _, M, _ = prob.run_batch(t_per_step * t_steps, t_steps, h, precision=precision)
    seq = np.stack([sequence_layout(M[b, :, :, 0, :], r3) for b in range(B)]).astype(np.float32)
    return seq, prob.last_stats


def write_database(path, sequence, field, intv=None):
    """Write the database arrays: HDF5 datasets ``sequence`` and ``field`` (attribute
    ``intv``) as the reference when h5py is importable, otherwise the same arrays
    in an .npz file.  Returns the path written."""
    path = Path(path)
    try:
        import h5py
    except ImportError:
        h5py = None
    if h5py is not None:
        out = path.with_suffix(".h5")
        with h5py.File(out, "w") as db:
            db.create_dataset("sequence", data=np.asarray(sequence, dtype=np.float32))
            db.create_dataset("field", data=np.asarray(field, dtype=np.float32))
            if intv is not None:
                db.attrs["intv"] = list(intv)
        return out
    out = path.with_suffix(".npz")
    extra = {} if intv is None else {"intv": np.asarray(intv)}
    np.savez(out, sequence=np.asarray(sequence, dtype=np.float32), field=np.asarray(field, dtype=np.float32),
             **extra)
    return out


def db_std_prob_4(datapath, n_seq, res, grid_size=(500e-9, 500e-9, 3e-9), t_steps=500, t_per_step=4e-12,
                  h_ext_a=(0, 360), h_ext_n=(0, 50), seed=0, intv=None, name=None, m0_state=None,
                  precision="int8"):
    """The whole database of db_std_prob_4 in one batched run: s-state (computed,
    or ``m0_state``), seeded fields, sequences, written under ``datapath``."""
    lo, hi = (0, n_seq) if intv is None else intv
    fname = name if name is not None else f"{n_seq}_{t_steps}_{res[0]}_{res[1]}_{lo}_{hi}"
    st = s_state(res, grid_size) if m0_state is None else np.asarray(m0_state)
    fields = std_prob_4_fields(n_seq, h_ext_a, h_ext_n, seed, (lo, hi))
    seq, _ = std_prob_4_sequences(st, res, fields, grid_size, t_steps, t_per_step, precision)
    return write_database(Path(datapath) / fname, seq, fields, (lo, hi))
