"""Exchange layout of the warp-row x pass (row variant 4), checked on the CPU.

The Stockham engine (specsim3d_b200/csrc/ss3d_engine.cuh) moves data between
radix passes through shared memory.  For tiles of one warp (fft_tile_regs with
SWM < 0) position p of row t sits at a ^ ((a >> 3) & 15), a = p * RPW + t.  This
file restates the engine's schedule (radix-8 passes, then one radix-4 or
radix-2 pass; butterfly jb of a pass reads jb + r N/R and writes
(jb/Ns) Ns R + jb mod Ns + r Ns) and the lane layout of rows_warp_body (lane =
c * RPW + t, c the rank of the lane in its row, jb = c + TPC m), and checks that
the layout is a permutation of each warp's slice and that every exchange
access of an FP32 tile (8-byte elements) needs the minimum number of
shared-memory wavefronts: 32 banks of 4 bytes, a 64-bit access served per
half-warp, so 2 wavefronts per warp instruction when conflict-free.
"""
import pytest


def radices(logn):
    n8, rem = logn // 3, logn % 3
    return [8] * n8 + ([4 if rem == 2 else 2] if rem else [])


def xidx(p, t, rpw):
    a = p * rpw + t
    return a ^ ((a >> 3) & 15)


def exchange_accesses(logn, et):
    """Positions (p, t) per lane of every shared-memory load and store of the
    exchanges, one list of 32 per warp instruction."""
    n = 1 << logn
    tpc = n // et
    rpw = 32 // tpc
    out = []
    ns = 1
    rad = radices(logn)
    for P, R in enumerate(rad):
        nbt = et // R
        if P > 0:                                   # loads of pass P
            for m in range(nbt):
                for r in range(R):
                    out.append([((lane // rpw) + tpc * m + r * (n // R), lane % rpw) for lane in range(32)])
        if P < len(rad) - 1:                        # stores of pass P
            for m in range(nbt):
                for r in range(R):
                    lanes = []
                    for lane in range(32):
                        jb = lane // rpw + tpc * m
                        lanes.append(((jb // ns) * ns * R + jb % ns + r * ns, lane % rpw))
                    out.append(lanes)
        ns *= R
    return out, rpw


def wavefronts_8byte(slots):
    """Wavefronts of one warp access of 8-byte elements at the given slot indices."""
    total = 0
    for half in (slots[:16], slots[16:]):
        words = {}
        for s in set(half):
            for w in (2 * s, 2 * s + 1):
                words.setdefault(w % 32, set()).add(w)
        total += max(len(v) for v in words.values())
    return total


@pytest.mark.parametrize("logn,et", [(5, 8), (6, 8), (7, 8), (8, 8), (9, 16)])
def test_warp_row_exchange_layout(logn, et):
    acc, rpw = exchange_accesses(logn, et)
    n = 1 << logn
    addrs = [xidx(p, t, rpw) for p in range(n) for t in range(rpw)]
    assert sorted(addrs) == list(range(n * rpw))          # a permutation of the warp's slice
    assert acc, "lengths of two or more passes exchange through shared memory"
    for lanes in acc:
        assert wavefronts_8byte([xidx(p, t, rpw) for p, t in lanes]) == 2


def test_plain_row_major_layout_conflicts():
    """Without the XOR the pass-0 stores of a length-256 row (positions 8 c + r)
    fall into 2 bank groups: the check above is not vacuous."""
    acc, rpw = exchange_accesses(8, 8)
    worst = max(wavefronts_8byte([p * rpw + t for p, t in lanes]) for lanes in acc)
    assert worst > 2
