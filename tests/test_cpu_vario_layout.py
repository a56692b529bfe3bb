"""CPU restatement of the variogram kernel's work layout (ss3d_vario.cu).

The GPU kernel walks every direction as lines of unit march step, stages the
lines of a CTA in shared memory (one or two row segments) and lets each warp
accumulate 16 lags over register blocks of 8 bases.  This test replays that
index arithmetic lane by lane in numpy (lines, lane-local march, staged rows,
partner rows, masks, lag chunks) and checks that

  * every global read lies inside the field,
  * every shared-memory row read by a counted pair was staged, from the march
    index the pair needs, and every base block read stays inside the allocation,
  * the pair sums give the oracle's gamma (f90:405-431) to 1e-12,

on the shapes and directions of the GPU tests, lines longer than one CTA
(several base blocks, the two-segment layout) and more than 128 lags.
"""
import numpy as np
import pytest

import oracle_lib as ora

VT, VB, VL, VNW, VP = 256, 8, 16, 8, 33
VLCH = VNW * VL


def floordiv(a, b):
    return a // b


def ceildiv(a, b):
    return -((-a) // b)


def geometry(n, s):
    """VarioGeo of ss3d_vario (host part), as a dict."""
    nx, ny, nz = n
    a, b, c = s
    lead = c if c != 0 else (b if b != 0 else a)
    if lead < 0:
        a, b, c = -a, -b, -c
    G = dict(nx=nx, ny=ny, nz=nz, sx=a, sy=b, sz=c, ncta=0)
    if a == 0 and b == 0 and c == 0:
        return G
    if b == 0 and c == 0:
        G.update(mode=1, sig=min(a, nx), mmax=(nx + a - 1) // a, nqx=(ny + 31) // 32, nqb=nz)
        ncta = G["nqx"] * nz * G["sig"]
    else:
        ax = 2 if c != 0 else 1
        sig = c if c != 0 else b
        na = nz if ax == 2 else ny
        sbv = b if ax == 2 else c
        nbv = ny if ax == 2 else nz
        mmax = (na + sig - 1) // sig
        mm1 = mmax - 1
        qx_lo, qx_hi = -mm1 * max(a, 0), nx - 1 + mm1 * max(-a, 0)
        qb_lo, qb_hi = -mm1 * max(sbv, 0), nbv - 1 + mm1 * max(-sbv, 0)
        G.update(mode=0, a=ax, sig=sig, mmax=mmax, qx_lo=qx_lo, nqx=(qx_hi - qx_lo + 1 + 31) // 32, qb_lo=qb_lo,
                 nqb=qb_hi - qb_lo + 1)
        ncta = G["nqx"] * G["nqb"] * sig
    G["tb"] = min(VT, (G["mmax"] + VB - 1) // VB * VB)
    G["nmb"] = (G["mmax"] + G["tb"] - 1) // G["tb"]
    G["ncta"] = ncta * G["nmb"]
    return G


def window(G, l0, nlag):
    nl = min(VLCH, nlag - l0 + 1)
    nw = (nl + VL - 1) // VL
    span = min(G["tb"] + nw * VL - 1, max(0, G["mmax"] - l0))
    one = min(G["mmax"], l0 + span)
    if one <= G["tb"] + span:
        W = dict(na=one, nb=0, pofs=l0, prow=max(0, one - l0))
    else:
        W = dict(na=G["tb"], nb=span, pofs=G["tb"], prow=span)
    W.update(l0=l0, nl=nl, nw=nw, rows=W["na"] + W["nb"] + VB)
    return W


def lane_line(G, cta, t):
    """(len, base, step, m0) of lane t of CTA cta."""
    mb = cta % G["nmb"]
    rest = cta // G["nmb"]
    m0 = mb * G["tb"]
    hi = G["mmax"]
    if G["mode"] == 1:
        jt = rest % G["nqx"]
        rest //= G["nqx"]
        k = rest % G["nqb"]
        rho = rest // G["nqb"]
        x0, y0, z0, dx, dy, dz = rho, jt * 32 + t, k, G["sx"], 0, 0
    else:
        xt = rest % G["nqx"]
        rest //= G["nqx"]
        qb = G["qb_lo"] + rest % G["nqb"]
        r = rest // G["nqb"]
        x0 = G["qx_lo"] + xt * 32 + t
        y0, z0 = (qb, r) if G["a"] == 2 else (r, qb)
        dx, dy, dz = G["sx"], G["sy"], G["sz"]
    lo = 0
    for c0, dc, n in ((x0, dx, G["nx"]), (y0, dy, G["ny"]), (z0, dz, G["nz"])):
        if dc == 0:
            if c0 < 0 or c0 >= n:
                hi = lo
        elif dc > 0:
            lo = max(lo, ceildiv(-c0, dc))
            hi = min(hi, floordiv(n - 1 - c0, dc) + 1)
        else:
            e = -dc
            lo = max(lo, ceildiv(c0 - n + 1, e))
            hi = min(hi, floordiv(c0, e) + 1)
    hi = max(hi, lo)
    ln = hi - lo
    step = dx + G["nx"] * (dy + G["ny"] * dz)
    base = x0 + G["nx"] * (y0 + G["ny"] * z0) + lo * step if ln > 0 else 0
    return ln, base, step, m0


def emulate(f, n, s, nlag):
    """gamma (nlag,) of one field f (nz, ny, nx) through the kernel layout."""
    G = geometry(n, s)
    flat = f.ravel()
    M = flat.size
    sums = np.zeros(nlag)
    if G["ncta"] == 0:
        return sums
    for l0 in range(1, nlag + 1, VLCH):
        W = window(G, l0, nlag)
        for cta in range(G["ncta"]):
            lines = [lane_line(G, cta, t) for t in range(32)]
            m0 = lines[0][3]
            smem = np.zeros((W["rows"], 32))
            src = np.full((W["rows"], 32), -1, dtype=np.int64)    # march index staged per row, -1 none
            for t, (ln, base, step, _) in enumerate(lines):
                for q in range(W["na"] + W["nb"]):
                    m = m0 + q if q < W["na"] else m0 + W["l0"] + (q - W["na"])
                    if m < ln:
                        idx = base + m * step
                        assert 0 <= idx < M
                        smem[q, t] = flat[idx]
                        src[q, t] = m
            ln_t = np.array([ln for ln, _, _, _ in lines])
            plim = np.minimum(ln_t - m0 - W["l0"], W["prow"])
            for w in range(W["nw"]):
                lw = w * VL
                bmax = min(G["tb"], int(plim.max()) - lw)
                acc = np.zeros((VL, 32))
                for b0 in range(0, max(bmax, 0), VB):
                    assert b0 + VB - 1 < W["rows"]
                    bv = smem[b0:b0 + VB]
                    q0 = b0 + lw
                    for p in range(VB + VL - 1):
                        ok = (q0 + p) < plim
                        if not ok.any():
                            continue
                        row = W["pofs"] + q0 + p
                        assert row < W["na"] + W["nb"]
                        for i in range(max(0, p - VL + 1), min(p, VB - 1) + 1):
                            j = p - i
                            b = b0 + i
                            # the pair (base b, lag l0 + lw + j) of lane t
                            assert (src[b, ok] == m0 + b).all()
                            assert (src[row, ok] == m0 + W["l0"] + b + lw + j).all()
                            d = smem[row] - bv[i]
                            acc[j] += np.where(ok, d * d, 0.0)
                for j in range(VL):
                    if lw + j < W["nl"]:
                        sums[l0 - 1 + lw + j] += acc[j].sum()
    nx, ny, nz = n
    out = np.zeros(nlag)
    for l in range(1, nlag + 1):
        npair = ora.npair_count(n, (l * s[0], l * s[1], l * s[2]))
        out[l - 1] = 0.5 * sums[l - 1] / npair if npair > 0 else 0.0
    return out


DIRS = [(1, 1, 0, 9), (1, -1, 0, 9), (0, 0, 1, 6), (2, 0, 0, 8), (-1, 0, 0, 5), (0, -1, 0, 7), (1, 2, -1, 4),
        (0, 3, 2, 3), (-2, 1, 1, 5), (0, 0, 0, 2), (40, 0, 0, 2)]


@pytest.mark.parametrize("shape", [(7, 13, 21), (1, 17, 33), (12, 1, 40), (5, 6, 1), (24, 24, 24)])
def test_layout_matches_oracle(shape):
    rng = np.random.default_rng(sum(shape))
    f = rng.normal(size=shape)
    n = (shape[2], shape[1], shape[0])
    ref = ora.vario(f[None], DIRS)[0]
    for k, (sx, sy, sz, nl) in enumerate(DIRS):
        got = emulate(f, n, (sx, sy, sz), nl)
        assert np.allclose(got, ref[k, :nl], rtol=1e-12, atol=1e-14), (sx, sy, sz)


@pytest.mark.parametrize("shape,dirs", [
    ((2, 3, 300), [(1, 0, 0, 299), (3, 0, 0, 99), (1, 1, 0, 2)]),       # three lag chunks, residues
    ((1, 1, 700), [(1, 0, 0, 200)]),                                    # three base blocks per line
    ((300, 2, 2), [(0, 0, 1, 140), (1, 0, 1, 20)]),                      # long z lines
])
def test_long_lines_and_many_lags(shape, dirs):
    rng = np.random.default_rng(11)
    f = rng.normal(size=shape)
    n = (shape[2], shape[1], shape[0])
    ref = ora.vario(f[None], dirs)[0]
    for k, (sx, sy, sz, nl) in enumerate(dirs):
        got = emulate(f, n, (sx, sy, sz), nl)
        assert np.allclose(got, ref[k, :nl], rtol=1e-12, atol=1e-14), (sx, sy, sz)


def test_both_row_layouts_are_exercised():
    """The cases above reach the one-segment layout and, for lags past one CTA's
    base range, the two-segment layout."""
    G = geometry((300, 3, 2), (1, 0, 0))
    assert window(G, 1, 299)["nb"] == 0
    assert window(G, 257, 299)["nb"] > 0
