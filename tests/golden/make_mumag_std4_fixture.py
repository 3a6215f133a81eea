"""Generates tests/golden/mumag_std4_published.npz from the reference's own
known-answer data for muMAG standard problem 4: the band of published
solutions that its std-problem-4 workflow loads and plots next to its own
result (matlab/examples/Micromagnetism/mumag_micromag_Std_problem_4/
Standard_problem_4.m:187-205, Published_solutions_field{1,2}.mat).  Each file
holds ``mean_avg`` and ``err`` of shape (1, 1000, 3): the mean and the spread
of the published <M_i>/Ms at 1000 times evenly spaced over [0, 1] ns.

Usage: python tests/golden/make_mumag_std4_fixture.py <MagTense source root>
"""
import sys
from pathlib import Path

import numpy as np
import scipy.io

if len(sys.argv) != 2:
    sys.exit(__doc__)
src = Path(sys.argv[1]) / "matlab" / "examples" / "Micromagnetism" / "mumag_micromag_Std_problem_4"
out = {"t_ns": np.linspace(0.0, 1.0, 1000)}
for field in (1, 2):
    d = scipy.io.loadmat(src / f"Published_solutions_field{field}.mat")
    out[f"field{field}_mean"] = np.asarray(d["mean_avg"], dtype=np.float64)[0]
    out[f"field{field}_err"] = np.asarray(d["err"], dtype=np.float64)[0]
np.savez_compressed(Path(__file__).with_name("mumag_std4_published.npz"), **out)
print({k: v.shape for k, v in out.items()})
