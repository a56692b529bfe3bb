"""Generate tests/golden/reference_pins.json from the reference's committed results.

The reference repository ships no .bin outputs, but it ships numbers computed
from seeded runs of the Fortran program:
  * docs/figures/scaling_cached.json  RMS variogram error of realization 1,
    full double precision (make_figures.py measure_scaling recipe:
    spherical 20/10/5 N45E, ipad 1, seed 99, n^3 grid, nreal 2 (1 at 256));
  * docs/figures/tables/figS1_yao_rms.csv, fig04_models_rms.csv,
    fig05_cases.csv, fig07_legacy_vs_padded.csv  statistics at 4-5 digits;
  * docs/figures/tables/fig12_conditional_validation.csv,
    fig13_conditional_nscore.csv  statistics of seeded conditional runs
    (make_figures.py cond_case / fig12_cond_validation / fig13_cond_nscore).
Each pin records the case that produced it so the tests can rerun it through
the oracle and through the CUDA path.  Run from the repository root:

    python tests/golden/make_golden.py /path/to/reference
"""
import csv
import json
import os
import sys

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_pins.json")


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    REF = sys.argv[1]
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
    for row in csv.DictReader(open(os.path.join(tab, "fig12_conditional_validation.csv"))):
        if row["code"] == "SPECSIM3D":
            pins["fig12"] = {k: (row[k] if k == "code" else float(row[k])) for k in row}
    pins["fig05"] = [dict(case=row["case"], model=row["model"], n_lags=int(row["n_lags"]), rms=float(row["rms"]),
                          mc_noise=float(row["mc_noise"]), rms_over_noise=float(row["rms_over_noise"]),
                          bias=float(row["bias"]))
                     for row in csv.DictReader(open(os.path.join(tab, "fig05_cases.csv")))]
    pins["fig13"] = {row["quantity"]: float(row["value"])
                     for row in csv.DictReader(open(os.path.join(tab, "fig13_conditional_nscore.csv")))}
    pins["cases"] = {
        "scaling": "grid n^3, d=1, spherical sill 1 ranges 20/10/5 az 45, nugget 0, seed 99, ipad 1; rms = mean over "
                   "directions (1,1,0),(1,-1,0),(0,0,1) with lags 1..int(a), a = 20,10,5, of the RMS of the numpy "
                   "variogram of realization 1 (float32 .bin) minus 1 - rho_sph(h/a)",
        "figS1": "64x64x16, spherical 20/10/5 az 45, seed 31791191, nreal 20, ipad 1, --vario dirs (1,1,0,40),"
                 "(1,-1,0,40),(0,0,1,10); rms/max of gamma_mean - gamma_model where gamma_model < 0.95",
        "fig04": "as figS1 for models 1,2,3 (ranges 20/10/5 az 45); rms over lags with h <= range of the direction",
        "fig07": "gaussian 20/10/5 az 45 nreal 40 seed 31791191, vario (1,1,0,57), mean gamma for h > 25 (ipad 0/1); "
                 "spherical nreal 300 seed 777: sd over realizations of the sample variance and mean (ipad 0/1)",
        "fig05": "64x64x16, ipad 1, seed 2024, nreal 20; 6 anisotropy cases x 3 models + nested sph/exp with nugget "
                 "0.1; --vario with 1,500 one-lag directions drawn by default_rng(12345).integers(-30..30, -30..30, "
                 "-12..12) (zero vectors dropped); gamma_model/mean/sd as printed (es14.6); lags with 0.05 < "
                 "gamma_model/sill < 0.97, first 300; rms, noise = rms of sd/sqrt(20), ratio, bias",
        "fig12": "64x64x16, exponential 20/10/5 az 45, nugget 0, ipad 1; truth = realization 1 of seed 2024 (.bin, "
                 "float32); 150 distinct nodes drawn by default_rng(7).choice(65536, 150, replace=False) in "
                 "(x, y, z) C order, data = truth there written with %.8g; conditioning cpar: columns 1 2 3 4 0, "
                 "trimming +-1e21, itrans 0 skmean 0, radii 30/15/8, angles 45/0/0, ndmax 24; 200 realizations of "
                 "seed 777 (.bin); statistics against exact simple kriging with all 150 data (ridge 1e-10)",
        "fig13": "as fig12 for truth and data locations; truth_ln = exp(1 + 0.8 truth), data = truth_ln at the "
                 "nodes (%.8g), itrans 1, zmin 0, zmax = 2 max(data), linear tails; 50 realizations of seed 99",
    }
    json.dump(pins, open(OUT, "w"), indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
