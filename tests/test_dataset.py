"""Std-problem-4 dataset driver (magtense_b200/dataset.py), host side: the
seeded fields are the reference's draws (database.py:62-70, restated here as
its per-sequence loop), the layout transform puts cell (ix, iy) of component a
at [t, a, ix, iy], and the database round-trips through its file."""
import numpy as np


def reference_field_loop(n_seq, seed, intv=None, h_ext_a=(0, 360), h_ext_n=(0, 50)):
    """database.py:58-70 restated: the interval's sequence i takes row i of the
    seeded table, for i in range(intv[1] - intv[0])."""
    if intv is None:
        intv = [0, n_seq]
    n_intv = intv[1] - intv[0]
    rng = np.random.default_rng(seed)
    rnd_mat = rng.random(size=(n_seq, 2))
    out = np.zeros((n_intv, 3))
    for i in range(n_intv):
        d = (h_ext_n[1] - h_ext_n[0]) * rnd_mat[i, 0] + h_ext_n[0]
        theta = np.deg2rad((h_ext_a[1] - h_ext_a[0]) * rnd_mat[i, 1] + h_ext_a[0])
        out[i, :2] = d * np.array([np.cos(theta), np.sin(theta)])
    return out


def test_fields_are_the_reference_draws():
    from magtense_b200.dataset import std_prob_4_fields
    n_seq, seed = 7, 3
    np.testing.assert_array_equal(std_prob_4_fields(n_seq, seed=seed), reference_field_loop(n_seq, seed))
    np.testing.assert_array_equal(std_prob_4_fields(n_seq, seed=seed, intv=(0, 4)),
                                  reference_field_loop(n_seq, seed, (0, 4)))
    # an interval that starts past 0 reuses the table's first rows, as the reference does
    got = std_prob_4_fields(n_seq, seed=seed, intv=(2, 5))
    np.testing.assert_array_equal(got, reference_field_loop(n_seq, seed, (2, 5)))
    np.testing.assert_array_equal(got, std_prob_4_fields(n_seq, seed=seed)[:3])
    np.testing.assert_array_equal(std_prob_4_fields(9, seed=5, h_ext_a=(10, 20), h_ext_n=(5, 6), intv=(4, 9)),
                                  reference_field_loop(9, 5, (4, 9), (10, 20), (5, 6)))


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
