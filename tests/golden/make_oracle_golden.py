"""Regression fixtures of the CPU oracle on the ``tiny`` system.

    python tests/golden/make_oracle_golden.py

Stores the seeded inputs' checksum and the oracle's outputs for three solver
settings, so any later change of the oracle's arithmetic is caught.  The
fixed-iteration case stops after 5 PCG steps: on this system the iterate of
band 1 between steps 7 and 10 is ill-conditioned (a one-ulp change of the
input moves it by up to 1e-8), so a cut there would compare rounding noise.  These
fixtures come from the oracle itself (the reference cannot run here); the
reference-side pins are in reference_pins.json.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import west_oracle as O  # noqa: E402
from west_b200.system import build_system, perturbations  # noqa: E402

s = build_system("tiny")
dvg = perturbations(s, 3, seed=7)
out = {"dvg": dvg, "evc": s.evc, "et": s.et, "vrs_sum": s.vrs.sum(), "alpha_pv": s.alpha_pv}
for tag, tr2, maxit in (("lite", -1.0, 250), ("tr2_1e-12", 1e-12, 250), ("fixed5", 0.0, 5)):
    dng, ierr = O.apply_operator(s, dvg, tr2, maxiter=maxit)
    out["dng_" + tag] = dng
    out["ierr_" + tag] = ierr
np.savez_compressed(os.path.join(HERE, "oracle_tiny.npz"), **out)
print("written", sorted(out))
