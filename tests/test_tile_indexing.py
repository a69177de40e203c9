"""CPU restatement of the index arithmetic of the tiled kernels, checked for
the invariants the kernels rely on (no GPU needed):

* 3D marching kernel (stage_fast.cu): in the k-edge tiles every lane's
  NTB-tap row reads columns inside the shared row, and the taps of an owned
  closure or interior row lie inside the block; every (j, k) column has
  exactly one owning tile; halo nodes map to the right shared columns;
* face-node kernel: every node on a block face is handled exactly once;
* return-map pass: its threads cover the interior nodes exactly once;
* 2D marching kernel (stage_fast2d.cu): the same per-lane rows and
  ownership in j, the halo columns, the y-face nodes stashed only in the
  tiles whose batch pass finishes them, and work items covering every
  (row, tile) once.

Tile sizes are read from the kernel sources, so the checks follow them."""

import itertools
import os
import re

import pytest

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "fdfault_b200", "csrc")


def _const(fname, pattern):
    with open(os.path.join(CSRC, fname)) as fh:
        m = re.search(pattern, fh.read())
    assert m, (fname, pattern)
    return tuple(int(g) for g in m.groups())


TJ, TK = _const("stage_fast.cu", r"constexpr int TJ = (\d+), TK = (\d+), NT = TJ \* TK;")
(TJ2,) = _const("stage_fast2d.cu", r"constexpr int TJ2 = (\d+);")
(KB2,) = _const("stage_fast2d.cu", r"constexpr int KB2 = (\d+);")


def lane_row(k, k0, n2, own, H):
    """(kb, ks, kmax, kw) of a lane in an edge tile (k_fast3d / tile2d)."""
    NB, NTB = 2 * H, 3 * H
    kb, ks, kmax, kw = k - k0, 1, 2 * H, 0
    if own and k < NB:
        kb, kmax, kw = H - k0, NTB - 1, (k + 1) * NTB
    elif own and k >= n2 - NB:
        kb, ks, kmax, kw = (n2 - 1 - k0) + H, -1, NTB - 1, (NB + n2 - k) * NTB
    return kb, ks, kmax, kw


def tiles(n, T):
    """(tile index, first node, is last) of the shifted-last-tile decomposition."""
    nt = (n + T - 1) // T
    return [(t, n - T if t == nt - 1 else t * T, t == nt - 1) for t in range(nt)]


def owns(x, t, last, n, T, NB):
    return last if x >= n - NB else (x // T == t)


def check_edge_rows(n, T, order):
    H = order - 1
    NB, NTB, VW = 2 * H, 3 * H, T + 2 * H
    owner = {}
    for t, x0, last in tiles(n, T):
        assert x0 >= 0
        edge = t == 0 or last
        for lane in range(T):
            x = x0 + lane
            assert 0 <= x < n
            own = owns(x, t, last, n, T, NB)
            if own:
                assert x not in owner
                owner[x] = t
            kb, ks, kmax, kw = lane_row(x, x0, n, own, H)
            assert 0 <= kw and kw + NTB <= (2 * NB + 1) * NTB
            if not edge:
                continue
            for tap in range(NTB):
                col = kb + ks * min(tap, kmax)
                assert 0 <= col < VW, (n, t, lane, tap, col)
                xx = x0 - H + col
                if own:   # an owned row reads only nodes of the block
                    assert 0 <= xx < n, (n, t, lane, tap, xx)
    assert sorted(owner) == list(range(n))


@pytest.mark.parametrize("order", [2, 3, 4])
def test_3d_k_edge_rows_and_ownership(order):
    for n2 in list(range(TK, TK + 70)) + [201, 208, 301, 401]:
        check_edge_rows(n2, TK, order)


@pytest.mark.parametrize("order", [2, 3, 4])
def test_3d_j_ownership(order):
    H = order - 1
    for n1 in list(range(TJ, TJ + 40)) + [201, 301]:
        owner = {}
        for t, j0, last in tiles(n1, TJ):
            for tj in range(TJ):
                j = j0 + tj
                if owns(j, t, last, n1, TJ, 2 * H):
                    assert j not in owner
                    owner[j] = t
        assert sorted(owner) == list(range(n1))


def test_3d_halo_columns():
    H = 3
    HN = 2 * H * (TK + TJ)
    assert HN <= TJ * TK
    seen = set()
    for tid in range(HN):
        if tid < 2 * H * TK:
            r, c = tid // TK, tid % TK
            hj, hk, kind = (r - H) if r < H else (TJ + r - H), c, 0
        else:
            t2 = tid - 2 * H * TK
            r, c = t2 // (2 * H), t2 % (2 * H)
            hj, hk, kind = r, (c - H) if c < H else (TK + c - H), 1
        # j-halo nodes lie above or below the tile rows, k-halo nodes left or right of its columns
        if kind == 0:
            assert (hj < 0 or hj >= TJ) and 0 <= hk < TK
            assert 0 <= hj + H < TJ + 2 * H
        else:
            assert 0 <= hj < TJ and (hk < 0 or hk >= TK)
            assert 0 <= hk + H < TK + 2 * H
        assert (kind, hj, hk) not in seen
        seen.add((kind, hj, hk))


def face_nodes_handled(n):
    """Nodes handled by k_faces3d: grid (ceil(max(n2, n1)/32), ceil(max(n0, n1)/4), 6) of 32 x 4."""
    n0, n1, n2 = n
    gx, gy = (max(n2, n1) + 31) // 32, (max(n0, n1) + 3) // 4
    out = []
    for fc in range(6):
        d = fc >> 1
        nb = n1 if d == 2 else n2
        na = n1 if d == 0 else n0
        for by, bx, ty, tx in itertools.product(range(gy), range(gx), range(4), range(32)):
            ub, ua = bx * 32 + tx, by * 4 + ty
            if ub >= nb or ua >= na:
                continue
            at = (n[d] - 1) if fc & 1 else 0
            i, j, k = (at, ua, ub) if d == 0 else ((ua, at, ub) if d == 1 else (ua, ub, at))
            if d >= 1 and i in (0, n0 - 1):
                continue
            if d == 2 and j in (0, n1 - 1):
                continue
            out.append((i, j, k))
    return out


@pytest.mark.parametrize("n", [(13, 8, 32), (25, 13, 37), (17, 40, 33), (30, 9, 70)])
def test_face_kernel_covers_each_face_node_once(n):
    got = face_nodes_handled(n)
    assert len(got) == len(set(got))
    want = {p for p in itertools.product(*[range(x) for x in n])
            if any(p[q] in (0, n[q] - 1) for q in range(3))}
    assert set(got) == want


@pytest.mark.parametrize("n", [(13, 8, 32), (25, 13, 37), (9, 10, 40)])
def test_return_map_pass_covers_interior_once(n):
    n0, n1, n2 = n
    n1i, n2i = n1 - 2, n2 - 2
    got = []
    for t in range((n0 - 2) * n1i * n2i):
        k, j, i = 1 + t % n2i, 1 + (t // n2i) % n1i, 1 + t // (n2i * n1i)
        got.append((i, j, k))
    assert len(set(got)) == len(got)
    assert set(got) == set(itertools.product(range(1, n0 - 1), range(1, n1 - 1), range(1, n2 - 1)))


@pytest.mark.parametrize("order", [2, 3, 4])
def test_2d_y_rows_ownership_halo_and_stash(order):
    H = order - 1
    NB, VW = 2 * H, TJ2 + 2 * H
    for n1 in list(range(TJ2, TJ2 + 60)) + [201, 401]:
        check_edge_rows(n1, TJ2, order)
        ntj = (n1 + TJ2 - 1) // TJ2
        for jt, j0, last in tiles(n1, TJ2):
            for lane in range(2 * H):
                hj = (j0 - H + lane) if lane < H else (j0 + TJ2 + lane - H)
                hcol = lane if lane < H else TJ2 + lane
                assert 0 <= hcol < VW and j0 - H + hcol == hj
            for lane in range(TJ2):
                j = j0 + lane
                own = owns(j, jt, last, n1, TJ2, NB)
                # a y-face node is stashed only where the batch pass finishes it
                if own and j == 0:
                    assert jt == 0
                if own and j == n1 - 1:
                    assert jt == ntj - 1
    assert 2 * KB2 == 32   # the batch pass: one lane per (row, side)


def test_2d_work_items_cover_rows_once():
    for n0, n1 in [(13, 32), (61, 40), (401, 201), (801, 401), (33, 64)]:
        ntj = (n1 + TJ2 - 1) // TJ2
        want, nsm = 8 * 148 * 16, 148
        chunks = (want + ntj - 1) // ntj
        chunk = max((n0 + chunks - 1) // chunks, 32)
        chunks = (n0 + chunk - 1) // chunk
        seen = set()
        for item in range(ntj * chunks):
            jt, ch = item % ntj, item // ntj
            ib, ie = ch * chunk, min(n0, ch * chunk + chunk)
            assert ib < ie
            for i in range(ib, ie):
                assert (i, jt) not in seen
                seen.add((i, jt))
        assert len(seen) == n0 * ntj
