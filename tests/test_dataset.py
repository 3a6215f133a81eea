"""Std-problem-4 dataset driver (magtense_b200/dataset.py), host side: the
seeded fields are the reference's draws (database.py:62-70, restated here as
its per-sequence loop), the layout transform puts cell (ix, iy) of component a
at [t, a, ix, iy], and the database round-trips through its file."""
import numpy as np


def test_fields_are_the_reference_draws():
    from magtense_b200.dataset import std_prob_4_fields
    n_seq, seed = 7, 3
    rng = np.random.default_rng(seed)
    rnd = rng.random(size=(n_seq, 2))
    want = np.zeros((n_seq, 3))
    for i in range(n_seq):
        d = (50 - 0) * rnd[i, 0] + 0
        theta = np.deg2rad((360 - 0) * rnd[i, 1] + 0)
        want[i, :2] = d * np.array([np.cos(theta), np.sin(theta)])
    np.testing.assert_array_equal(std_prob_4_fields(n_seq, seed=seed), want)
    np.testing.assert_array_equal(std_prob_4_fields(n_seq, seed=seed, intv=(2, 5)), want[2:5])


def test_sequence_layout():
    from magtense_b200.dataset import sequence_layout
    res = (5, 3, 1)
    t, n = 4, 15
    M = np.random.default_rng(0).standard_normal((t, n, 3))
    seq = sequence_layout(M, res)
    assert seq.shape == (t, 3, 5, 3)
    for ix in range(5):
        for iy in range(3):
            np.testing.assert_array_equal(seq[:, :, ix, iy], M[:, iy * res[0] + ix, :])


def test_database_round_trip(tmp_path):
    from magtense_b200.dataset import write_database
    seq = np.random.default_rng(1).standard_normal((2, 4, 3, 5, 3)).astype(np.float32)
    field = np.arange(6, dtype=np.float32).reshape(2, 3)
    out = write_database(tmp_path / "db", seq, field, (0, 2))
    if out.suffix == ".npz":
        z = np.load(out)
        np.testing.assert_array_equal(z["sequence"], seq)
        np.testing.assert_array_equal(z["field"], field)
        np.testing.assert_array_equal(z["intv"], [0, 2])
    else:
        import h5py
        with h5py.File(out) as db:
            np.testing.assert_array_equal(db["sequence"][...], seq)
