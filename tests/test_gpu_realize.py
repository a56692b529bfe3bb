"""GPU parity of the spectrum and the realization path against the CPU oracle.

Bars (stated per test):
  * Park-Miller states: bit-exact, every coefficient, several realizations.
  * FP64 spectrum amplitudes: 1e-12 of max amp (different FFT order).
  * FP64 realizations: max |gpu - oracle| <= 1e-9 * sqrt(C0) (the FFT
    algorithms differ in rounding order; spectral values that sit at the FP64
    noise floor of the forward FFT give the remaining difference).
  * FP32 realizations: max |gpu - oracle| <= 1e-5 * sqrt(C0), the precision-form
    target.
"""
import numpy as np
import pytest

import oracle_lib as ora
import recipes

pytestmark = pytest.mark.gpu

CASES = [
    # (n, structs, nugget, d, ipad)
    ((64, 64, 16), [(1, 1.0, 20.0, 10.0, 5.0, 45.0, 0.0, 0.0)], 0.0, (1.0, 1.0, 1.0), 1),       # cfg1 model
    ((30, 20, 9), [(2, 0.7, 12.0, 6.0, 3.0, 30.0, 10.0, 5.0)], 0.3, (1.0, 1.5, 0.5), 1),        # odd, anisotropic
    ((17, 33, 1), [(3, 1.0, 8.0, 4.0, 4.0, 120.0, 0.0, 0.0)], 0.1, (1.0, 1.0, 1.0), 1),         # 2D
    ((16, 16, 16), [(2, 1.0, 5.0, 5.0, 5.0, 0.0, 0.0, 0.0)], 0.0, (1.0, 1.0, 1.0), 0),          # compact ipad 0
    ((12, 7, 5), [(1, 0.5, 6.0, 3.0, 2.0, 300.0, -20.0, 15.0), (2, 0.4, 3.0, 3.0, 1.0, 0, 0, 0)], 0.1,
     (1.0, 1.0, 1.0), 0),                                                                       # nested, ipad 0
    ((1, 24, 10), [(2, 1.0, 6.0, 3.0, 2.0, 0.0, 0.0, 0.0)], 0.0, (1.0, 1.0, 1.0), 0),           # npx = 1
]


def _expected_states(full, np3):
    """First-draw state per half-spectrum index: own draw, or the partner's draw."""
    npx, npy, npz = np3
    h = npx // 2 + 1 if npx >= 2 else 1
    k, j, i = np.meshgrid(np.arange(npz), np.arange(npy), np.arange(h), indexing="ij")
    own = full[k, j, i]
    part = full[(npz - k) % npz, (npy - j) % npy, (npx - i) % npx]
    return np.where(own != 0, own, part)


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("igauss", [0, 1])
def test_rng_states_bit_exact(gpu, case, igauss):
    n, sts, nug, d, ipad = CASES[case]
    sp = gpu.Spectrum(sts, nug, d, n, ipad)
    iseed = 69069 + 7 * case
    full = ora.fill_states(sp.np, iseed, 3, igauss)
    for r in range(3):
        exp = _expected_states(full[r], sp.np)
        got = sp.debug_states(iseed, r, igauss).astype(np.int64)
        assert np.array_equal(got, exp), f"realization {r}: {np.count_nonzero(got != exp)} states differ"


@pytest.mark.parametrize("case", range(len(CASES)))
def test_spectrum_fp64(gpu, case):
    n, sts, nug, d, ipad = CASES[case]
    sp = gpu.Spectrum(sts, nug, d, n, ipad)
    np3, rc = ora.grid(sts, d, n, ipad)
    assert rc == 0 and tuple(np3) == sp.np
    amp_o, st_o = ora.spectrum(sts, nug, d, sp.np)
    amp_g = sp.amp()
    ref = recipes.half_of_full(amp_o, sp.np[0])
    assert np.max(np.abs(amp_g - ref)) <= 1e-12 * np.max(ref)
    assert sp.stats["c0"] == st_o["c0"]
    assert abs(sp.stats["spos"] - st_o["spos"]) <= 1e-12 * st_o["spos"]
    assert abs(sp.stats["sneg"] - st_o["sneg"]) <= 1e-12 * st_o["spos"]
    assert abs(sp.stats["maxreal"] - st_o["maxreal"]) <= 1e-12 * st_o["maxreal"]


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("igauss", [0, 1])
def test_coefficients_fp64(gpu, case, igauss):
    n, sts, nug, d, ipad = CASES[case]
    sp = gpu.Spectrum(sts, nug, d, n, ipad)
    amp_o, _ = ora.spectrum(sts, nug, d, sp.np)
    iseed = 4711 + case
    for r in (0, 1):
        co = recipes.half_of_full(ora.coefficients(amp_o, sp.np, iseed, r, igauss), sp.np[0])
        cg = sp.debug_coefficients(iseed, r, igauss, gpu.FP64)
        scale = max(np.max(np.abs(co)), 1e-300)
        assert np.max(np.abs(cg - co)) <= 1e-12 * scale


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("igauss", [0, 1])
def test_realize_fp64_vs_oracle(gpu, case, igauss):
    n, sts, nug, d, ipad = CASES[case]
    sp = gpu.Spectrum(sts, nug, d, n, ipad)
    amp_o, st = ora.spectrum(sts, nug, d, sp.np)
    iseed, nreal = 1234 + case, 3
    res_o, zs_o = ora.realize(amp_o, sp.np, n, iseed, nreal, igauss)
    res_g, zs_g = sp.realize(iseed, nreal, igauss, gpu.FP64, zstats=True)
    c0 = st["c0"]
    err = np.max(np.abs(res_g - res_o))
    assert err <= 1e-9 * np.sqrt(c0), err
    assert np.allclose(zs_g[:, :2], zs_o[:, :2], rtol=0, atol=1e-9)


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("igauss", [0, 1])
def test_realize_fp32_vs_oracle(gpu, case, igauss):
    n, sts, nug, d, ipad = CASES[case]
    sp = gpu.Spectrum(sts, nug, d, n, ipad)
    amp_o, st = ora.spectrum(sts, nug, d, sp.np)
    iseed, nreal = 99 + case, 2
    res_o, _ = ora.realize(amp_o, sp.np, n, iseed, nreal, igauss)
    res_g = sp.realize(iseed, nreal, igauss, gpu.FP32, dtype=np.float32)
    err = np.max(np.abs(res_g.astype(np.float64) - res_o)) / np.sqrt(st["c0"])
    assert err <= 1e-5, err


def test_sharding_is_exact(gpu):
    n, sts, nug, d, ipad = CASES[1]
    sp = gpu.Spectrum(sts, nug, d, n, ipad)
    for prec in (gpu.FP64, gpu.FP32):
        full = sp.realize(555, 5, 1, prec)
        for r0, k in ((0, 2), (2, 3), (4, 1), (1, 3)):
            part = sp.realize(555, k, 1, prec, r_first=r0)
            assert np.array_equal(part, full[r0:r0 + k])


def test_device_output_matches_host(gpu):
    import torch
    n, sts, nug, d, ipad = CASES[0]
    sp = gpu.Spectrum(sts, nug, d, n, ipad)
    host = sp.realize(31, 2, 0, gpu.FP32, dtype=np.float32)
    dev = torch.empty((2, n[2], n[1], n[0]), dtype=torch.float32, device="cuda")
    sp.realize(31, 2, 0, gpu.FP32, out=dev)
    torch.cuda.synchronize()
    assert np.array_equal(dev.cpu().numpy(), host)


@pytest.mark.parametrize("n", [32, 64])
def test_golden_scaling_rms(gpu, n):
    """Reference-published RMS of realization 1 (docs/figures/scaling_cached.json)."""
    import json
    import os
    pins = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_pins.json")))
    want = [p for p in pins["scaling_rms"] if p["n"] == n][0]
    c = recipes.scaling_case(n)
    sp = gpu.Spectrum(c["structs"], c["nugget"], c["d"], c["n"], c["ipad"])
    assert list(sp.np) == want["periodic"]
    res = sp.realize(c["seed"], 1, 0, gpu.FP64, dtype=np.float32)
    rms = recipes.scaling_rms(res[0])
    assert abs(rms - want["rms"]) <= 1e-9 * want["rms"], (rms, want["rms"])


def test_tile_variants_give_identical_results(gpu):
    """All tile variants run the same butterflies: outputs are bitwise identical."""
    from specsim3d_b200 import _lib
    L = _lib.lib()
    n, sts, nug, d, ipad = CASES[0]                   # periodic 128 x 128 x 32
    sp = gpu.Spectrum(sts, nug, d, n, ipad)
    for prec in (gpu.FP32, gpu.FP64):
        ref = sp.realize(77, 2, 1, prec)
        for v in (1, 2, 3, 4):
            for kind, logn in ((0, 7), (1, 5), (2, 6)):
                assert L.ss3d_set_variant(kind, prec, logn, v if kind == 2 or v < 4 else 0) == 0
            assert np.array_equal(sp.realize(77, 2, 1, prec), ref)
        for kind, logn in ((0, 7), (1, 5), (2, 6)):
            L.ss3d_set_variant(kind, prec, logn, 0)
    chosen = gpu.autotune(sp, 1, gpu.FP32, 2)
    assert chosen["row_pass"] in set(range(7)) and set(chosen.values()) <= set(range(10))
    assert np.array_equal(sp.realize(77, 2, 1, gpu.FP32), sp.realize(77, 2, 1, gpu.FP32))


def _kinds_of(np3):
    """(kind, log2 length) of the column passes of a periodic grid."""
    lg = [int(v).bit_length() - 1 for v in np3]
    if np3[2] > 1:
        return [(1, lg[2])] + ([(0, lg[1])] if np3[1] > 1 else [])
    return [(1, lg[1])] if np3[1] > 1 else []


@pytest.mark.parametrize("igauss", [0, 1])
@pytest.mark.parametrize("n,ipad", [((40, 36, 20), 1), ((64, 64, 16), 1), ((33, 17, 1), 1), ((1, 24, 12), 1),
                                     ((100, 1, 30), 1), ((24, 12, 40), 1), ((4, 4, 200), 1), ((8, 200, 4), 1),
                                     ((20, 70, 9), 0)])
def test_two_line_variants_identical(gpu, n, ipad, igauss):
    """FP32 column passes with two adjacent lines per thread (packed FP32
    instructions, variants 4-7) give the bits of the one-line tiles, including
    grids whose half-spectrum rows end in a padding element, 2D grids whose
    synthesis runs along y, and columns of 512 (pruned one-line tiles against
    unpruned two-line tiles) and of 64 positions."""
    from specsim3d_b200 import _lib
    L = _lib.lib()
    sts = [(2, 0.8, 14.0, 9.0, 5.0, 35.0, 10.0, 5.0)]
    sp = gpu.Spectrum(sts, 0.2, (1.0, 1.0, 1.0), n, ipad)
    kinds = [(k, lg) for k, lg in _kinds_of(sp.np) if 5 <= lg <= 10]
    if not kinds:
        pytest.skip("no tuned column length on this grid")
    ref = sp.realize(4321, 3, igauss, gpu.FP32, dtype=np.float32)
    try:
        for v in (4, 5, 6, 7):
            for kind, lg in kinds:
                assert L.ss3d_set_variant(kind, gpu.FP32, lg, v) == 0
            got = sp.realize(4321, 3, igauss, gpu.FP32, dtype=np.float32)
            assert np.array_equal(got, ref), (v, float(np.max(np.abs(got - ref))))
        # mixed: synthesis on two lines, middle pass on one, and the reverse;
        # middle pass 8 and 9: tiles staged by bulk tensor copies
        for vs, vm in ((4, 0), (0, 6), (5, 1), (7, 5), (0, 8), (6, 9), (4, 8)):
            for kind, lg in kinds:
                L.ss3d_set_variant(kind, gpu.FP32, lg, vs if kind == 1 else vm)
            assert np.array_equal(sp.realize(4321, 3, igauss, gpu.FP32, dtype=np.float32), ref)
    finally:
        for kind, lg in kinds:
            L.ss3d_set_variant(kind, gpu.FP32, lg, 0)
    assert L.ss3d_set_variant(2, gpu.FP32, 6, 7) != 0      # the row pass has no two-line tiles
    assert L.ss3d_set_variant(1, gpu.FP32, 6, 8) != 0      # bulk-copy tiles: middle pass only
    assert L.ss3d_set_variant(0, gpu.FP32, 6, 10) != 0


@pytest.mark.parametrize("prec", ["FP32", "FP64"])
@pytest.mark.parametrize("n", [(40, 36, 20), (256, 3, 2), (33, 17, 1), (100, 1, 30), (101, 3, 5), (200, 9, 7),
                               (600, 2, 1)])
def test_row_warp_variant_identical(gpu, n, prec):
    """Row pass variant 4 (each row in the registers of one warp, packing by
    shuffles) gives the bits of the shared-memory row tiles, for odd and even
    nx, row counts that leave a block partly empty, row lengths 32..512, and
    the same mean / variance table."""
    from specsim3d_b200 import _lib
    L = _lib.lib()
    P = getattr(gpu, prec)
    sts = [(1, 0.9, 12.0, 7.0, 4.0, 20.0, 0.0, 0.0)]
    sp = gpu.Spectrum(sts, 0.1, (1.0, 1.0, 1.0), n, 1)
    lg = int(sp.np[0]).bit_length() - 2                 # log2 of the row transform length npx/2
    if not 5 <= lg <= 10:
        pytest.skip("row length outside the tuned range")
    ref, zref = sp.realize(99, 3, 1, P, dtype=np.float32, zstats=True)
    try:
        assert L.ss3d_set_variant(2, P, lg, 4) == 0
        got, zgot = sp.realize(99, 3, 1, P, dtype=np.float32, zstats=True)
    finally:
        L.ss3d_set_variant(2, P, lg, 0)
    assert np.array_equal(got, ref), float(np.max(np.abs(got - ref)))
    assert np.allclose(zgot, zref, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("n", [(40, 36, 20), (256, 3, 2), (33, 17, 1), (100, 1, 30), (101, 3, 5), (200, 9, 7),
                               (120, 7, 3), (600, 2, 1), (256, 256, 9)])
def test_row_pair_variant_identical(gpu, n):
    """Row pass variant 6 (FP32: two rows per lane on packed FP32) gives the
    bits of the one-row kernels, for odd and even nx, odd row counts (a pair
    that straddles two planes, a last row without a partner), row lengths
    32..256 and, past them, the variant 4 fallback (npx 1024); float32 and
    float64 outputs, the mean / variance table, and through a batch."""
    import torch
    from specsim3d_b200 import _lib
    L = _lib.lib()
    sts = [(2, 0.9, 12.0, 7.0, 4.0, 20.0, 0.0, 0.0)]
    sp = gpu.Spectrum(sts, 0.1, (1.0, 1.0, 1.0), n, 1)
    lg = int(sp.np[0]).bit_length() - 2
    if not 5 <= lg <= 10:
        pytest.skip("row length outside the tuned range")
    ref, zref = sp.realize(4321, 3, 1, gpu.FP32, dtype=np.float32, zstats=True)
    ref64 = sp.realize(4321, 3, 1, gpu.FP32, dtype=np.float64)
    try:
        assert L.ss3d_set_variant(2, gpu.FP32, lg, 6) == 0
        got, zgot = sp.realize(4321, 3, 1, gpu.FP32, dtype=np.float32, zstats=True)
        got64 = sp.realize(4321, 3, 1, gpu.FP32, dtype=np.float64)
        out = torch.empty((3, n[2], n[1], n[0]), dtype=torch.float32, device="cuda")
        b = gpu.Batch([(sp, 4321, 1, 0, 3, out)])
        b.run()
        b.close()
        gotb = out.cpu().numpy()
    finally:
        L.ss3d_set_variant(2, gpu.FP32, lg, 0)
    sp.close()
    assert np.array_equal(got, ref), float(np.max(np.abs(got - ref)))
    assert np.array_equal(got64, ref64)
    assert np.array_equal(gotb, ref)
    assert np.allclose(zgot, zref, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("case", [0, 1, 2])
@pytest.mark.parametrize("igauss", [0, 1])
def test_coefficients_fp32(gpu, case, igauss):
    """FP32 synthesis: hardware sine/cosine after an exact integer quarter-turn
    reduction, series logarithm near u = 1; every coefficient within 2e-6 of
    the largest against the oracle's FP64 values."""
    n, sts, nug, d, ipad = CASES[case]
    sp = gpu.Spectrum(sts, nug, d, n, ipad)
    amp_o, _ = ora.spectrum(sts, nug, d, sp.np)
    co = recipes.half_of_full(ora.coefficients(amp_o, sp.np, 8080 + case, 1, igauss), sp.np[0])
    cg = sp.debug_coefficients(8080 + case, 1, igauss, gpu.FP32)
    assert np.max(np.abs(cg - co)) <= 2e-6 * np.max(np.abs(co))


def test_fp32_error_at_full_size(gpu):
    """Precision form at the bench's full size (256^3 on 512^3, gaussian model):
    every cell within 1e-5 sqrt(C0) of the FP64 path.  The origin cell sums every
    coefficient with phase 1, so a systematic bias of the FP32 phasor shows up
    there even when it is invisible on small grids."""
    import torch
    n = (256, 256, 256)
    sp = gpu.Spectrum([(3, 1.0, 60.0, 30.0, 15.0, 30.0, 20.0, 10.0)], 0.1, (1.0, 1.0, 1.0), n, 1)
    o32 = torch.empty((2, 256, 256, 256), dtype=torch.float32, device="cuda")
    o64 = torch.empty((2, 256, 256, 256), dtype=torch.float64, device="cuda")
    for igauss in (1, 0):
        sp.realize(12345, 2, igauss, gpu.FP32, out=o32)
        sp.realize(12345, 2, igauss, gpu.FP64, out=o64)
        torch.cuda.synchronize()
        err = float((o32.double() - o64).abs().amax().item()) / np.sqrt(sp.stats["c0"])
        assert err <= 1e-5, (igauss, err)


def test_misaligned_device_output_is_refused(gpu):
    """Rows of even length are stored as 2-element vectors: a device output that
    starts off a pair boundary (a contiguous view at an odd element offset) is
    refused by ss3d_realize and ss3d_batch_create before any kernel runs, and
    the memory stays untouched.  Host outputs have no alignment rule."""
    import torch
    n, sts, nug, d, ipad = CASES[0]
    sp = gpu.Spectrum(sts, nug, d, n, ipad)
    M = n[0] * n[1] * n[2]
    for dt in (torch.float32, torch.float64):
        flat = torch.zeros(M + 1, dtype=dt, device="cuda")
        view = flat[1:].view(1, n[2], n[1], n[0])
        with pytest.raises(gpu.SpecsimError, match="multiple of"):
            sp.realize(7, 1, 0, gpu.FP32, out=view)
        torch.cuda.synchronize()
        assert float(flat.abs().sum().item()) == 0.0
    flat = torch.zeros(M + 1, dtype=torch.float32, device="cuda")
    with pytest.raises(gpu.SpecsimError, match="multiple of"):
        gpu.Batch([(sp, 7, 0, 0, 1, flat[1:].view(1, n[2], n[1], n[0]))])
    host = np.zeros(M + 1, dtype=np.float32)
    got = sp.realize(7, 1, 0, gpu.FP32, out=host[1:].reshape(1, n[2], n[1], n[0]))
    assert np.array_equal(got, sp.realize(7, 1, 0, gpu.FP32, dtype=np.float32))
    sp.close()


@pytest.mark.parametrize("n", [(64, 64, 16), (256, 256, 8), (40, 36, 20), (30, 20, 9), (128, 100, 3)])
def test_bulk_copy_middle_pass_identical(gpu, n):
    """Middle pass variants 8 and 9 (tiles staged in shared memory by bulk
    tensor copies, two-stage pipeline in a persistent CTA) give the bits of the
    direct-load tiles, through ss3d_realize (several realizations per launch),
    and the batched form (graph capture) on the same grid."""
    import torch
    from specsim3d_b200 import _lib
    L = _lib.lib()
    sts = [(3, 1.0, 14.0, 9.0, 5.0, 35.0, 10.0, 5.0)]
    sp = gpu.Spectrum(sts, 0.1, (1.0, 1.0, 1.0), n, 1)
    if sp.np[2] == 1 or sp.np[1] == 1:
        pytest.skip("no middle pass on this grid")
    lg = int(sp.np[1]).bit_length() - 1
    if not 5 <= lg <= 10:
        pytest.skip("middle-pass length outside the tuned range")
    ref = sp.realize(2468, 3, 1, gpu.FP32, dtype=np.float32)
    try:
        for v in (8, 9):
            assert L.ss3d_set_variant(0, gpu.FP32, lg, v) == 0
            got = sp.realize(2468, 3, 1, gpu.FP32, dtype=np.float32)
            assert np.array_equal(got, ref), (v, float(np.max(np.abs(got - ref))))
            out = torch.empty((3, n[2], n[1], n[0]), dtype=torch.float32, device="cuda")
            b = gpu.Batch([(sp, 2468, 1, 0, 3, out)])
            b.run()
            b.close()
            assert np.array_equal(out.cpu().numpy(), ref)
    finally:
        L.ss3d_set_variant(0, gpu.FP32, lg, 0)


@pytest.mark.parametrize("n", [(256, 256, 16), (200, 180, 9), (100, 64, 20), (300, 256, 5), (64, 40, 30),
                               (256, 256, 256)])
def test_fused_middle_row_pass_identical(gpu, n):
    """Row variant 5 (FP32): the middle (y) and row (x) passes of a plane in one
    thread-block cluster, the y output handed to the row tiles through
    distributed shared memory, gives the bits of the separate passes, per call
    and batched, for cluster sizes 2..8 (rows per CTA times CTAs >= ny) and
    row lengths 256..1024."""
    import torch
    from specsim3d_b200 import _lib
    L = _lib.lib()
    sts = [(2, 1.0, 30.0, 12.0, 6.0, 20.0, 5.0, 0.0)]
    sp = gpu.Spectrum(sts, 0.05, (1.0, 1.0, 1.0), n, 1)
    lx = int(sp.np[0]).bit_length() - 2
    ly = int(sp.np[1]).bit_length() - 1
    if not (7 <= lx <= 9 and 6 <= ly <= 9 and sp.np[2] > 1):
        pytest.skip(f"periodic grid {sp.np} outside the fused pass's lengths")
    k = 2 if n[2] > 64 else 3
    ref = sp.realize(97531, k, 1, gpu.FP32, dtype=np.float32)
    try:
        assert L.ss3d_set_variant(2, gpu.FP32, lx, 5) == 0
        got = sp.realize(97531, k, 1, gpu.FP32, dtype=np.float32)
        assert np.array_equal(got, ref), float(np.max(np.abs(got - ref)))
        out = torch.empty((k, n[2], n[1], n[0]), dtype=torch.float32, device="cuda")
        b = gpu.Batch([(sp, 97531, 1, 0, k, out)])
        b.run()
        b.close()
        assert np.array_equal(out.cpu().numpy(), ref)
        # statistics requested: the separate passes run, same values
        got2, zs = sp.realize(97531, k, 1, gpu.FP32, dtype=np.float32, zstats=True)
        assert np.array_equal(got2, ref)
    finally:
        L.ss3d_set_variant(2, gpu.FP32, lx, 0)
    sp.close()


def test_preload_kernels(gpu):
    """ss3d_preload_kernels loads every kernel of the library's modules (a
    second call finds them loaded); realizations are the same after it."""
    n, sts, nug, d, ipad = CASES[1]
    sp = gpu.Spectrum(sts, nug, d, n, ipad)
    before = sp.realize(2718, 2, 1, gpu.FP32)
    gpu.preload_kernels()
    gpu.preload_kernels()
    assert np.array_equal(sp.realize(2718, 2, 1, gpu.FP32), before)
    sp.close()
