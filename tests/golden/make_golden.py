"""Generate tests/golden/reference_pins.json from the reference's committed results.

The reference repository ships no .bin outputs, but it ships numbers computed
from seeded runs of the Fortran program:
  * docs/figures/scaling_cached.json  RMS variogram error of realization 1,
    full double precision (make_figures.py measure_scaling recipe:
    spherical 20/10/5 N45E, ipad 1, seed 99, n^3 grid, nreal 2 (1 at 256));
  * docs/figures/tables/figS1_yao_rms.csv, fig04_models_rms.csv,
    fig07_legacy_vs_padded.csv  statistics at 4-5 digits.
Each pin records the case that produced it so the tests can rerun it through
the oracle and through the CUDA path.  Run from the repository root:

    python tests/golden/make_golden.py /path/to/reference
"""
import csv
import json
import os
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_pins.json")


def main():
    sc = json.load(open(os.path.join(REF, "docs/figures/scaling_cached.json")))
    pins = {"scaling_rms": [], "figS1": [], "fig04": [], "fig07": []}
    for k, v in sc.items():
        if k.startswith("specsim3d_"):
            pins["scaling_rms"].append(dict(n=v["n"], nreal=v["nreal"], periodic=v["periodic"], rms=v["rms"],
                                            source="docs/figures/scaling_cached.json:" + k))
    tab = os.path.join(REF, "docs/figures/tables")
    for row in csv.DictReader(open(os.path.join(tab, "figS1_yao_rms.csv"))):
        pins["figS1"].append(dict(direction=row["direction"], rms=float(row["rms_mean_vs_model"]),
                                  maxerr=float(row["max_abs_error"])))
    for row in csv.DictReader(open(os.path.join(tab, "fig04_models_rms.csv"))):
        if row["method"] == "SPECSIM3D":
            pins["fig04"].append(dict(model=row["model"], direction=row["direction"],
                                      rms=float(row["rms_within_range"])))
    for row in csv.DictReader(open(os.path.join(tab, "fig07_legacy_vs_padded.csv"))):
        pins["fig07"].append(dict(case=row["case"], quantity=row["quantity"], value=float(row["value"])))
    pins["cases"] = {
        "scaling": "grid n^3, d=1, spherical sill 1 ranges 20/10/5 az 45, nugget 0, seed 99, ipad 1; rms = mean over "
                   "directions (1,1,0),(1,-1,0),(0,0,1) with lags 1..int(a), a = 20,10,5, of the RMS of the numpy "
                   "variogram of realization 1 (float32 .bin) minus 1 - rho_sph(h/a)",
        "figS1": "64x64x16, spherical 20/10/5 az 45, seed 31791191, nreal 20, ipad 1, --vario dirs (1,1,0,40),"
                 "(1,-1,0,40),(0,0,1,10); rms/max of gamma_mean - gamma_model where gamma_model < 0.95",
        "fig04": "as figS1 for models 1,2,3 (ranges 20/10/5 az 45); rms over lags with h <= range of the direction",
        "fig07": "gaussian 20/10/5 az 45 nreal 40 seed 31791191, vario (1,1,0,57), mean gamma for h > 25 (ipad 0/1); "
                 "spherical nreal 300 seed 777: sd over realizations of the sample variance and mean (ipad 0/1)",
    }
    json.dump(pins, open(OUT, "w"), indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
