"""Index invariants of the triangular solves' step-indexed tile-boundary rows
(xfp_solve.cu: row_base, the loaders' rj0/rk0).  Stored cells of a line run
from i = lo - ((lo + j + k) & 3) over a multiple of 4 cells (xfp_layout.cu),
so i lies in [-3, ni + 2].  A tile (J, K) of height NW owns R = ni_max + NW + 36
rows, row = step - row_base(J, K).  Checked here on the CPU, over real layouts,
for both directions:
  * every stored cell's publication row lies in [0, R);
  * the row a consumer reads for its step tau is the row its source tile
    published the source cell at (step tau - 1)."""
import numpy as np
import pytest

from xfluid_b200 import scenes


def _lines(mat):
    nk, nj, ni = mat.shape
    f = mat == 1
    out = {}
    for k in range(nk):
        for j in range(nj):
            idx = np.nonzero(f[k, j])[0]
            if len(idx):
                lo, hi = int(idx.min()), int(idx.max())
                Llo = lo - ((lo + j + k) & 3)
                out[(j, k)] = (Llo, ((hi + 1 - Llo) + 3) & ~3)
    return out


def _row_base(J, K, nw, ni, maxT, rev):
    lowest = 32 * J + nw * K - 3
    return maxT - (lowest + ni + nw + 35) if rev else lowest


def _step(i, j, k, maxT, rev):
    return maxT - (i + j + k) if rev else i + j + k


@pytest.mark.parametrize("shape,nw", [((24, 40, 70), 8), ((24, 40, 70), 15), ((20, 33, 45), 16)])
def test_rows_in_range_and_consumer_matches_producer(shape, nw):
    nk, nj, ni = shape
    mat = scenes.blob_scene(dims=(ni, nj, nk), seed=5, obstacle_frac=0.0, fractional=False).mat
    # fluid up to the ends of some lines (the padding then reaches i = -3 and ni + 2)
    mat[:, :, :3] = 1
    mat[:, :, -3:] = 1
    maxT, R = ni + nj + nk, ni + nw + 36
    L = _lines(mat)
    for rev in (False, True):
        for (j, k), (lo, ln) in L.items():
            J, K = j // 32, k // nw
            rb = _row_base(J, K, nw, ni, maxT, rev)
            for i in range(lo, lo + ln):
                row = _step(i, j, k, maxT, rev) - rb
                assert 0 <= row < R, (rev, i, j, k, row, R)
        # consumer side: the loader of tile (J, K) reads, for its step tau, the
        # row (tau - 1) - row_base(source tile); the source cell is the
        # neighbour at the same i one line back along j (or k)
        for (j, k), (lo, ln) in L.items():
            J, K = j // 32, k // nw
            for dj, dk in ((1, 0), (0, 1)):
                sj, sk = (j + dj, k + dk) if rev else (j - dj, k - dk)
                if (sj // 32, sk // nw) == (J, K) or (sj, sk) not in L:
                    continue          # same tile, or no source line
                slo, sln = L[(sj, sk)]
                SJ, SK = sj // 32, sk // nw
                rb_src = _row_base(SJ, SK, nw, ni, maxT, rev)
                for i in range(max(lo, slo), min(lo + ln, slo + sln)):
                    tau = _step(i, j, k, maxT, rev)
                    assert _step(i, sj, sk, maxT, rev) == tau - 1
                    assert (tau - 1) - rb_src == _step(i, sj, sk, maxT, rev) - rb_src
                    assert 0 <= (tau - 1) - rb_src < R
