"""The C ABI library on a machine without a GPU: it loads, exports every symbol
declared in include/specsim3d_gpu.h, and its host-side model logic (setrot,
covariance, ipad grid rule) agrees with the oracle bit for bit."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle_lib as ora

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "specsim3d_gpu.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ss3d_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from specsim3d_b200 import _lib
    L = _lib.lib()
    names = header_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(_lib.EXPORTS) <= set(names) | {"ss3d_realize_noalloc"}


def test_version_and_last_error():
    from specsim3d_b200 import _lib
    L = _lib.lib()
    assert b"sm_100a" in L.ss3d_version()
    assert isinstance(L.ss3d_last_error(), bytes)


def _random_structs(rng, nst):
    out = []
    for _ in range(nst):
        it = int(rng.integers(1, 4))
        a = np.sort(rng.uniform(1.0, 60.0, 3))[::-1]
        out.append((it, float(rng.uniform(0.1, 2.0)), float(a[0]), float(a[1]), float(a[2]),
                    float(rng.uniform(-90, 400)), float(rng.uniform(-60, 60)), float(rng.uniform(-90, 90))))
    return out


def test_setrot_bit_exact():
    import specsim3d_b200 as ss
    rng = np.random.default_rng(11)
    for _ in range(200):
        s = _random_structs(rng, 1)[0]
        rot, axes = ss.setrot(s)
        o = ora.structs([s])[0]
        assert np.array_equal(rot.ravel(), np.array(o.rot[:]))
        assert np.array_equal(axes.ravel(), np.array(o.axes[:]))


def test_covariance_bit_exact():
    import specsim3d_b200 as ss
    rng = np.random.default_rng(12)
    for _ in range(100):
        sts = _random_structs(rng, int(rng.integers(1, 4)))
        nug = float(rng.uniform(0, 0.3))
        o = ora.structs(sts)
        for _ in range(20):
            h = rng.integers(-30, 31, 3).astype(float) * rng.choice([0.5, 1.0, 2.5])
            c = ss.covariance(sts, nug, *h)
            assert c == ora.lib().ora_covariance(o, len(sts), nug, *h)
        c0 = nug
        for s in sts:
            c0 = c0 + s[1]
        assert ss.covariance(sts, nug, 0, 0, 0) == c0


def test_grid_rule_matches_oracle():
    import specsim3d_b200 as ss
    rng = np.random.default_rng(13)
    for _ in range(300):
        sts = _random_structs(rng, int(rng.integers(1, 4)))
        n = (int(rng.integers(1, 300)), int(rng.integers(1, 300)), int(rng.choice([1, int(rng.integers(1, 200))])))
        d = tuple(float(v) for v in rng.choice([0.5, 1.0, 2.0, 3.7], 3))
        ipad = int(rng.integers(0, 2))
        np3, rc = ora.grid(sts, d, n, ipad)
        if rc:
            with pytest.raises(Exception):
                ss.grid_size(sts, d, n, ipad)
        else:
            assert ss.grid_size(sts, d, n, ipad) == tuple(np3)


def test_baseline_configs_grids():
    """Periodic grids of the benchmark configurations."""
    import specsim3d_b200 as ss
    assert ss.grid_size([(1, 1.0, 20, 10, 5, 45, 0, 0)], (1, 1, 1), (64, 64, 16), 1) == (128, 128, 32)
    assert ss.grid_size([(3, 1.0, 60, 30, 15, 30, 20, 10)], (1, 1, 1), (256, 256, 256), 1) == (512, 512, 512)
    assert ss.grid_size([(2, 1.0, 40, 20, 8, 60, 0, 0)], (1, 1, 1), (128, 128, 64), 1) == (256, 256, 128)


def test_invalid_arguments_fail_loudly():
    import specsim3d_b200 as ss
    with pytest.raises(ss.SpecsimError, match="ranges must be positive"):
        ss.grid_size([(1, 1.0, 0.0, 10, 5, 0, 0, 0)], (1, 1, 1), (8, 8, 8), 1)
    with pytest.raises(ss.SpecsimError, match="nstruct"):
        ss.grid_size([], (1, 1, 1), (8, 8, 8), 1)
    with pytest.raises(ss.SpecsimError, match="too large"):
        ss.grid_size([(1, 1.0, 900, 900, 900, 0, 0, 0)], (1, 1, 1), (600, 600, 600), 1)


def test_gpu_calls_without_gpu_report_cuda_error():
    """No silent CPU fallback: on a machine without a GPU the compute entry points fail."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import specsim3d_b200 as ss
    with pytest.raises(ss.SpecsimError):
        ss.Spectrum([(1, 1.0, 5, 5, 5, 0, 0, 0)], 0.0, (1, 1, 1), (8, 8, 8), 1)


def test_variant_selection_ranges():
    """ss3d_set_variant (host only): 0-3 for every pass; 4-7 for the FP32 column
    passes (two lines per thread); 8-9 for the FP32 middle pass (tiles staged
    by bulk tensor copies); 4 for the row pass in both precisions (rows held in
    warps); anything else is refused."""
    from specsim3d_b200 import _lib
    import specsim3d_b200 as ss
    L = _lib.lib()
    try:
        for prec in (ss.FP32, ss.FP64):
            for kind in (0, 1, 2):
                for v in range(4):
                    assert L.ss3d_set_variant(kind, prec, 8, v) == 0
            assert L.ss3d_set_variant(2, prec, 8, 4) == 0
            assert (L.ss3d_set_variant(2, prec, 8, 5) == 0) == (prec == ss.FP32)   # fused middle + rows
            assert (L.ss3d_set_variant(2, prec, 8, 6) == 0) == (prec == ss.FP32)   # two rows per lane
            assert L.ss3d_set_variant(2, prec, 8, 7) != 0
            assert L.ss3d_set_variant(0, prec, 8, -1) != 0
            assert L.ss3d_set_variant(3, prec, 8, 0) != 0
        for kind in (0, 1):
            assert L.ss3d_set_variant(kind, ss.FP32, 8, 7) == 0
            assert L.ss3d_set_variant(kind, ss.FP64, 8, 4) != 0
        # middle pass only: 8, 9 stage their tiles with bulk tensor copies (FP32)
        assert L.ss3d_set_variant(0, ss.FP32, 8, 9) == 0
        assert L.ss3d_set_variant(0, ss.FP32, 8, 10) != 0
        assert L.ss3d_set_variant(1, ss.FP32, 8, 8) != 0
        assert L.ss3d_set_variant(0, ss.FP64, 8, 8) != 0
    finally:
        for prec in (ss.FP32, ss.FP64):
            for kind in (0, 1, 2):
                L.ss3d_set_variant(kind, prec, 8, 0)
