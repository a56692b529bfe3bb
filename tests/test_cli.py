"""The drop-in command line `specsim3d file.par [--vario f] [--gauss|--bin|--vtk|--cond f]`.

CPU tests: grammar errors give the reference's messages and exit codes (checked
beside the oracle's restatement of the Fortran driver).  GPU tests: the same
parameter files through our binary and through the oracle give the same
files; the checks of the reference's own scripts (tests/test_vario_fortran.py,
tests/test_gauss_amplitudes.py, tests/test_conditional.py) are restated with
our binary as the black box.
"""
import csv
import os
import subprocess

import numpy as np
import pytest

import oracle_lib as ora
import recipes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "specsim3d_b200", "bin", "specsim3d")
HEADER = "Parameters for SPECSIM3D\n************************\n\nSTART OF PARAMETERS:\n"


def run(exe, args, cwd):
    return subprocess.run([exe] + list(args), cwd=cwd, capture_output=True, text=True, timeout=600)


def write(path, text):
    with open(path, "w") as fh:
        fh.write(text)


BAD_FILES = {
    "bad_code.par": HEADER + "0 0 0\n1 1 1\n8 8 8\n0.0 1\n1 1.0 3 3 3 0 0 0\n1 1 1\nb\n1\n9\n0\n",
    "bad_nout.par": HEADER + "0 0 0\n1 1 1\n8 8 8\n0.0 1\n1 1.0 3 3 3 0 0 0\n1 1 1\nb\n10\n",
    "bad_icond.par": "0 0 0\n1 1 1\n8 8 8\n0.0 1\n1 1.0 3 3 3 0 0 0\n1 1 1\nb\n1\n3\n2\n",
    "bad_igauss.par": "0 0 0\n1 1 1\n8 8 8\n0.0 1\n1 1.0 3 3 3 0 0 0\n1 1 1 2\nb\n",
    "bad_range.par": "0 0 0\n1 1 1\n8 8 8\n0.0 1\n1 1.0 0 3 3 0 0 0\n1 1 1\nb\n",
    "bad_nst.par": "0 0 0\n1 1 1\n8 8 8\n0.0 11\n",
    "missing_code.par": "0 0 0\n1 1 1\n8 8 8\n0.0 1\n1 1.0 3 3 3 0 0 0\n1 1 1\nb\n2\n3\n",
    "huge.par": "0 0 0\n1 1 1\n600 600 600\n0.0 1\n1 1.0 300 300 300 0 0 0\n1 1 1\nb\n",
}


@pytest.mark.parametrize("name", sorted(BAD_FILES))
def test_grammar_errors_match_reference(tmp_path, name):
    ora.build()
    write(tmp_path / name, BAD_FILES[name])
    a = run(CLI, [name], tmp_path)
    b = run(ora.EXE, [name], tmp_path)
    assert a.returncode == b.returncode, (a.stdout, a.stderr, b.stdout, b.stderr)
    assert a.stdout.splitlines()[:1] == b.stdout.splitlines()[:1]
    assert a.stderr.strip().splitlines()[-1:] == b.stderr.strip().splitlines()[-1:]


def test_unknown_option_and_missing_file(tmp_path):
    a = run(CLI, ["nothere.par"], tmp_path)
    assert a.returncode == 1 and "Parameter file not found" in a.stdout
    write(tmp_path / "ok.par", BAD_FILES["bad_code.par"])
    a = run(CLI, ["ok.par", "--frobnicate"], tmp_path)
    assert a.returncode == 1 and "unknown option" in a.stdout


# ---------------------------------------------------------------- GPU
def _strip_times(out):
    return [l for l in out.splitlines() if "time" not in l]


def _bin(path, nreal, n):
    return np.fromfile(path, dtype="<f4").reshape(nreal, n[2], n[1], n[0])


@pytest.mark.gpu
def test_cfg1_files_and_stdout_match_oracle(tmp_path):
    """64x64x16 spherical 20/10/5 N45E, ipad 1, seed 69069: .bin, .vti, .out, .vtk and --vario CSV."""
    ora.build()
    par = HEADER + "0.5 0.5 0.5\n1 1 1\n64 64 16\n0.0 1\n1 1.0 20 10 5 45 0 0\n69069 2 1\ncfg1\n4\n1\n2\n3\n4\n0\n"
    write(tmp_path / "cfg1.par", par)
    write(tmp_path / "v.par", "3 1\n1 1 0 30\n1 -1 0 30\n0 0 1 30\n")
    os.mkdir(tmp_path / "o")
    write(tmp_path / "o" / "cfg1.par", par)
    write(tmp_path / "o" / "v.par", "3 1\n1 1 0 30\n1 -1 0 30\n0 0 1 30\n")
    a = run(CLI, ["cfg1.par", "--vario", "v.par"], tmp_path)
    b = run(ora.EXE, ["cfg1.par", "--vario", "v.par"], tmp_path / "o")
    assert a.returncode == 0, a.stdout + a.stderr
    assert b.returncode == 0
    la, lb = _strip_times(a.stdout), _strip_times(b.stdout)
    assert len(la) == len(lb)
    for x, y in zip(la, lb):
        if "max|Im|" in x or "Im S" in x:
            continue   # rounding-level diagnostics of the two FFTs
        assert x == y, (x, y)
    n = (64, 64, 16)
    fa, fb = _bin(tmp_path / "cfg1.bin", 2, n), _bin(tmp_path / "o" / "cfg1.bin", 2, n)
    assert np.max(np.abs(fa.astype(np.float64) - fb)) <= 1e-6
    # .vti arrays equal the .bin byte for byte (reference test_parameter_file_format)
    raw = open(tmp_path / "cfg1.vti", "rb").read()
    head = raw[:raw.index(b"<AppendedData")].decode()
    assert 'WholeExtent="0 63 0 63 0 15"' in head and head.count("<DataArray") == 2
    pos = raw.index(b"_", raw.index(b"<AppendedData")) + 1
    nb = 4 * 64 * 64 * 16
    for r in range(2):
        off = pos + r * (nb + 8)
        assert int.from_bytes(raw[off:off + 8], "little") == nb
        assert np.array_equal(np.frombuffer(raw[off + 8:off + 8 + nb], dtype="<f4"), fa[r].ravel())
    # the XML header is identical to the oracle's
    rawb = open(tmp_path / "o" / "cfg1.vti", "rb").read()
    assert raw[:pos] == rawb[:pos]
    # binary VTK: same header, big-endian data equal to the .bin
    for r in (1, 2):
        va = open(tmp_path / f"cfg1_{r}.vtk", "rb").read()
        vb = open(tmp_path / "o" / f"cfg1_{r}.vtk", "rb").read()
        ha = va[:va.index(b"LOOKUP_TABLE default\n") + 21]
        assert ha == vb[:len(ha)]
        assert np.array_equal(np.frombuffer(va[len(ha):len(ha) + nb], dtype=">f4"), fa[r - 1].ravel())
    # GSLIB .out: same header lines, values within the printed precision
    oa = open(tmp_path / "cfg1.out").read().splitlines()
    ob = open(tmp_path / "o" / "cfg1.out").read().splitlines()
    assert oa[:4] == ob[:4] and len(oa) == len(ob)
    va = np.array([[float(v) for v in l.split()] for l in oa[4:]])
    vb = np.array([[float(v) for v in l.split()] for l in ob[4:]])
    assert np.max(np.abs(va - vb)) <= 1e-6
    # variogram CSV: same header, pair counts exact, gammas within the es14.6 print
    ca = list(csv.reader(open(tmp_path / "cfg1_vario.csv")))
    cb = list(csv.reader(open(tmp_path / "o" / "cfg1_vario.csv")))
    assert ca[0] == cb[0] and len(ca) == len(cb)
    for x, y in zip(ca[1:], cb[1:]):
        assert x[:7] == y[:7]
        assert np.allclose([float(v) for v in x[7:]], [float(v) for v in y[7:]], rtol=2e-6, atol=1e-12)


@pytest.mark.gpu
def test_vario_fortran_script_checks(tmp_path):
    """Restatement of the reference's tests/test_vario_fortran.py against our binary."""
    nx, ny, nz, nreal, kmax = 64, 64, 16, 5, 40
    dirs = [(1, 1, 0), (1, -1, 0), (0, 0, 1)]
    write(tmp_path / "t.par", HEADER + f"0 0 0\n1 1 1\n{nx} {ny} {nz}\n0.0 1\n1 1.0 20 10 5 45 0 0\n31791191 {nreal} 1\n"
                                       "t_vario\n1\n3\n0\n")
    write(tmp_path / "v.par", f"{len(dirs)} 0\n" + "\n".join(f"{a} {b} {c} {kmax}" for a, b, c in dirs) + "\n")
    r = run(CLI, ["t.par", "--vario", "v.par"], tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    f = _bin(tmp_path / "t_vario.bin", nreal, (nx, ny, nz)).transpose(0, 3, 2, 1).astype(np.float64)
    rows = list(csv.reader(open(tmp_path / "t_vario_vario.csv")))[1:]
    worst = 0.0
    for d, step in enumerate(dirs, 1):
        ref = np.array([float(x[8]) for x in rows if int(x[0]) == d])
        g, _ = recipes.vario_shift(f, step, kmax)
        worst = max(worst, float(np.abs(g.mean(0)[:len(ref)] - ref).max()))
    assert worst <= 2e-6


@pytest.mark.gpu
def test_gauss_amplitudes_script_checks(tmp_path):
    """Restatement of the reference's tests/test_gauss_amplitudes.py (16^3 compact grid, 300 realizations)."""
    n, nreal = 16, 300

    def go(base, fourth="", flag=None):
        write(tmp_path / f"{base}.par", HEADER + f"0 0 0\n1 1 1\n{n} {n} {n}\n0.0 1\n2 1.0 5 5 5 0 0 0\n"
                                                 f"4711 {nreal} 0 {fourth}\n{base}\n1\n3\n0\n")
        r = run(CLI, [f"{base}.par"] + ([flag] if flag else []), tmp_path)
        assert r.returncode == 0, r.stdout + r.stderr
        return np.fromfile(tmp_path / f"{base}.bin", dtype=np.float32).reshape(nreal, n, n, n).astype(float), r.stdout

    fa, _ = go("a")
    fb, out = go("b", fourth="1")
    fc, _ = go("c", flag="--gauss")
    va, vb = fa.reshape(nreal, -1).var(axis=1), fb.reshape(nreal, -1).var(axis=1)
    assert va.std() < 1e-5
    assert vb.std() > 0.03
    assert abs(vb.mean() - va.mean()) < 4 * vb.std() / np.sqrt(nreal)

    def vx(f):
        return np.array([0.5 * np.mean((f[:, :, :, k:] - f[:, :, :, :-k]) ** 2) for k in range(1, 6)])
    assert np.abs(vx(fa) - vx(fb)).max() < 0.04
    z = fb.ravel() / fb.std()
    assert abs(np.mean(z ** 4) - 3.0) < 0.1
    assert np.array_equal(fb, fc)
    assert "Gaussian" in out


@pytest.mark.gpu
def test_conditional_script_checks(tmp_path):
    """Restatement of tests/test_conditional.py: data reproduced, nscore table, par-file block == legacy --cond."""
    from scipy.stats import norm
    nx, ny, nz, nreal = 30, 30, 10, 50
    rng = np.random.default_rng(3)
    idx = rng.choice(nx * ny * nz, 40, replace=False)
    i, j, k = np.unravel_index(idx, (nx, ny, nz))
    v = rng.normal(size=40)
    write(tmp_path / "tc_data.dat", "test data\n4\nx\ny\nz\nv\n" + "".join(
        " ".join("%.8g" % q for q in p) + "\n" for p in np.c_[i, j, k, v]))
    write(tmp_path / "tc.par", f"0 0 0\n1 1 1\n{nx} {ny} {nz}\n0.0 1\n1 1.0 12 8 6 30 0 0\n12345 {nreal} 1\ntc\n")
    cblock = "tc_data.dat\n1 2 3 4 0\n-1e21 1e21\n0 0.0\n-5 5\n1 0\n1 0\n100 100 100\n0 0 0\n100\n"
    write(tmp_path / "tc.cpar", cblock)
    r = run(CLI, ["tc.par", "--bin", "--cond", "tc.cpar"], tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    sims = _bin(tmp_path / "tc.bin", nreal, (nx, ny, nz))
    assert np.abs(sims[:, k, j, i] - v[None]).max() < 1e-5
    base = open(tmp_path / "tc.par").read().splitlines()
    new = base[:-1] + ["tc_new", "3", "3", "2", "4", "1"] + cblock.splitlines()
    write(tmp_path / "tc_new.par", "\n".join(new) + "\n")
    r = run(CLI, ["tc_new.par"], tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    assert open(tmp_path / "tc.bin", "rb").read() == open(tmp_path / "tc_new.bin", "rb").read()
    assert os.path.exists(tmp_path / f"tc_new_{nreal}.vtk")
    # nscore table and back transform, 2D lognormal data
    rng = np.random.default_rng(5)
    nd = 200
    idx = rng.choice(64 * 64, nd, replace=False)
    x, y = (idx % 64).astype(float), (idx // 64).astype(float)
    vv = np.exp(rng.normal(1.0, 0.8, nd))
    write(tmp_path / "tn_data.dat", "test data\n3\nx\ny\nv\n" + "".join(
        " ".join("%.8g" % q for q in p) + "\n" for p in np.c_[x, y, vv]))
    write(tmp_path / "tn.par", "0 0 0\n1 1 1\n64 64 1\n0.0 1\n2 1.0 15 15 15 0 0 0\n777 10 1\ntn\n")
    write(tmp_path / "tn.cpar", "tn_data.dat\n1 2 0 3 0\n0 1e21\n1 0.0\n0.0 200.0\n1 0\n1 0\n30 30 30\n0 0 0\n16\n")
    r = run(CLI, ["tn.par", "--bin", "--cond", "tn.cpar"], tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    table = np.loadtxt(tmp_path / "tn_nscore.trn", skiprows=4)
    assert np.abs(table[:, 1] - norm.ppf((np.arange(nd) + 0.5) / nd)).max() < 1e-6
    sims = np.fromfile(tmp_path / "tn.bin", dtype="<f4").reshape(10, 64, 64)
    assert np.abs(sims[:, idx // 64, idx % 64] - vv[None]).max() / vv.max() < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [[], ["--precision", "fp32"]])
def test_streamed_float32_outputs(tmp_path, prec):
    """Outputs that are all float32 files (.bin, .vti, binary VTK of every
    realization) are written by the streaming path: chunks realized straight to
    float32 and written by a second thread while the next chunk computes.  The
    files are the same bytes as the all-in-memory path (here forced by adding
    the GSLIB .out) and match the oracle's within float32 rounding; 40
    realizations of 64x64x16 make several chunks."""
    ora.build()
    base = HEADER + "0 0 0\n1 1 1\n64 64 16\n0.1 1\n2 1.0 12 6 4 30 10 0\n4711 40 1 1\n{b}\n{k}\n{codes}\n0\n"
    write(tmp_path / "s.par", base.format(b="s", k=3, codes="2\n3\n4"))
    write(tmp_path / "m.par", base.format(b="m", k=4, codes="1\n2\n3\n4"))
    a = run(CLI, ["s.par"] + prec, tmp_path)
    b = run(CLI, ["m.par"] + prec, tmp_path)
    assert a.returncode == 0 and b.returncode == 0, a.stdout + a.stderr + b.stdout + b.stderr
    la = [l for l in _strip_times(a.stdout) if "realization" in l]
    lb = [l for l in _strip_times(b.stdout) if "realization" in l]
    assert la == lb and len(la) == 40
    assert open(tmp_path / "s.bin", "rb").read() == open(tmp_path / "m.bin", "rb").read()
    va, vb = open(tmp_path / "s.vti", "rb").read(), open(tmp_path / "m.vti", "rb").read()
    assert va == vb
    for r in (1, 17, 40):
        assert open(tmp_path / f"s_{r}.vtk", "rb").read()[-1000:] == open(tmp_path / f"m_{r}.vtk", "rb").read()[-1000:]
    if not prec:
        os.mkdir(tmp_path / "o")
        write(tmp_path / "o" / "s.par", base.format(b="s", k=3, codes="2\n3\n4"))
        c = run(ora.EXE, ["s.par"], tmp_path / "o")
        assert c.returncode == 0
        fa = _bin(tmp_path / "s.bin", 40, (64, 64, 16)).astype(np.float64)
        fc = _bin(tmp_path / "o" / "s.bin", 40, (64, 64, 16)).astype(np.float64)
        assert np.max(np.abs(fa - fc)) <= 1e-6
