"""Extract the facts the reference's own regression data records about this
path into reference_pins.json.

Reads WEST's test-suite logs as text (test001: SiH4 in a cubic L=20 bohr cell
at 25 Ry, FFT 64^3) and its checker tolerances.  Run in a tree where the WEST
sources are available; the output is committed so the tests never read the
reference at run time:

    python tests/golden/make_reference_pins.py /path/to/West
"""
import json
import os
import sys

ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
w = json.load(open(os.path.join(ref, "test-suite/test001/ref/wstat.json")))
par = json.load(open(os.path.join(ref, "test-suite/parameters.json")))
ctl = w["input"]["wstat_control"]
pins = {
    "source": "test-suite/test001/ref/wstat.json, test-suite/parameters.json",
    "cell_alat_bohr": w["system"]["cell"]["alat"],
    "omega_bohr3": w["system"]["cell"]["omega"],
    "ecutwfc_ry": w["system"]["basis"]["ecutwfc:ry"],
    "npw_sum": w["system"]["basis"]["npw"]["sum"],
    "fft_s": w["system"]["3dfft"]["s"],
    "gamma_only": w["system"]["basis"]["gamma_only"],
    "tr2_dfpt": ctl["tr2_dfpt"],
    "n_pdep_eigen": ctl["n_pdep_eigen"],
    "n_pdep_times": ctl["n_pdep_times"],
    "n_dfpt_maxiter": ctl["n_dfpt_maxiter"],
    "trev_pdep": ctl["trev_pdep"],
    "trev_pdep_rel": ctl["trev_pdep_rel"],
    "davitr_dfpt_tr2": [d["dfpt_tr2"] for d in w["exec"]["davitr"]],
    "davitr_dav_iter": [d["dav_iter"] for d in w["exec"]["davitr"]],
    "davitr_dfpt_dim": [d["dfpt_dim"] for d in w["exec"]["davitr"]],
    "davitr_diago_dim": [d["diago_dim"] for d in w["exec"]["davitr"]],
    "davitr_notcnv": [d["notcnv"] for d in w["exec"]["davitr"]],
    "checker_pdep_eigenvalue_tol": par.get("tolerance", par).get("pdep_eigenvalue", None)
        if isinstance(par.get("tolerance", par), dict) else None,
}
out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_pins.json")
json.dump(pins, open(out, "w"), indent=1)
print(json.dumps(pins, indent=1))
