"""Generates tests/golden/fem_prism_normH.npz from the reference's own FEM
validation data for the rotated prism (COMSOL line graphs of |B| = mu0|H|):
documentation/examples_FEM_validation/Validation_prism/Validation_prism_normH_{x,y,z}.txt
of the MagTense project.  Every 8th point along each line is kept.

Usage: python tests/golden/make_fem_prism_fixture.py <MagTense source root>
"""
import sys
from pathlib import Path

import numpy as np

if len(sys.argv) != 2:
    sys.exit(__doc__)
root = Path(sys.argv[1])
src = root / "documentation" / "examples_FEM_validation" / "Validation_prism"
out = {}
for c in "xyz":
    T = np.loadtxt(src / f"Validation_prism_normH_{c}.txt", comments="%")
    out[f"line_{c}"] = T[::8].astype(np.float64)
np.savez_compressed(Path(__file__).with_name("fem_prism_normH.npz"), **out)
print({k: v.shape for k, v in out.items()})
