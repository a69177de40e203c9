"""CPU restatement of the index arithmetic that x slabs add to the stage
kernels, checked over the plans ``plan_slabs`` makes (no GPU needed):

* the marching kernel's chunks (stage_reg.cu launch_order / reg_march)
  cover each plane a slab updates exactly once, and every chunk either
  starts at a block face, starts past the closure rows (its x window is
  filled by the prefill path) or lies wholly in the closing rows, whose x
  derivatives come from the pre-pass;
* every plane a chunk, the reference-order kernel or a closure row reads
  is one the slab updates or one of its ghost planes;
* the reference-order kernel's thread index (stage_exact.cuh volume_node)
  and the return-map pass (stage_fast.cu k_return_map3) map onto the
  updated planes exactly once;
* the planes one slab packs are the planes its neighbour unpacks, inside
  the packing slab;
* each fault node of a y- or z-normal fault, and the whole of an x-normal
  one, is finished by exactly one slab."""

import itertools

import pytest

from fdfault_b200 import slabs


def pick_chunk(n0, tiles, slots, H):
    """stage_reg.cu pick_chunk."""
    best, bestcost = n0, 1 << 30
    for chunks in range(1, 65):
        chunk = (n0 + chunks - 1) // chunks
        if chunk < 16 and chunks > 1:
            break
        nc = (n0 + chunk - 1) // chunk
        waves = (tiles * nc + slots - 1) // slots
        cost = waves * (chunk + H + 1)
        if cost < bestcost:
            bestcost, best = cost, chunk
    return best


def block_ranges(blocks, x0, x1):
    """solver.cpp set_x_range: (lo, n, xb, xe) per x block."""
    out = []
    for lo, n in blocks:
        xb = min(max(x0 - lo, 0), n)
        xe = min(max(x1 - lo, 0), n)
        out.append((lo, n, xb, max(xe, xb)))
    return out


LAYOUTS = [
    ([(0, 401)], 2), ([(0, 401)], 8), ([(0, 401)], 25), ([(0, 72)], 3),
    ([(0, 40), (40, 40)], 2), ([(0, 100), (100, 60), (160, 120)], 5), ([(0, 601)], 7),
]


@pytest.mark.parametrize("blocks,world", LAYOUTS)
@pytest.mark.parametrize("order", [2, 3, 4])
@pytest.mark.parametrize("tiles,slots", [(199, 296), (14, 296), (2, 296)])
def test_chunks_cover_updated_planes_and_read_inside_the_slab(blocks, world, order, tiles, slots):
    H = order - 1
    NB, NTB = 2 * H, 3 * H
    nx = sum(n for _, n in blocks)
    plan = slabs.plan_slabs(blocks, world)
    for x0, x1 in plan:
        readable = set(range(max(x0 - H, 0), min(x1 + H, nx)))
        for lo, n0, xb, xe in block_ranges(blocks, x0, x1):
            nown = xe - xb
            if nown <= 0:
                continue
            chunk = pick_chunk(nown, tiles, slots, H)
            nchunks = (nown + chunk - 1) // chunk
            seen = []
            for z in range(nchunks):
                ib = xb + z * chunk
                ie = min(xe, ib + chunk)
                assert ib < ie
                seen.extend(range(ib, ie))
                prefill = NB <= ib < n0 - NB
                assert ib == 0 or prefill or ib >= n0 - NB, (ib, n0)
                # planes the chunk reads: its window (prefill or inserts) and leading planes
                first = ib - H if prefill else ib
                reads = range(first, min(ie + H, n0))
                for i in reads:
                    assert lo + i in readable, (x0, x1, lo + i)
                # closure rows of planes this chunk updates: taps 0..NTB-1 from the face
                for i in range(ib, ie):
                    if i < NB:
                        assert all(lo + t in readable for t in range(NTB))
                    elif i >= n0 - NB:
                        assert all(lo + n0 - 1 - t in readable for t in range(NTB))
            assert seen == list(range(xb, xe))


@pytest.mark.parametrize("blocks,world", LAYOUTS[:5])
def test_reference_order_threads_and_return_map_cover_updated_planes(blocks, world):
    n1, n2 = 3, 4
    for x0, x1 in slabs.plan_slabs(blocks, world):
        for lo, n0, xb, xe in block_ranges(blocks, x0, x1):
            got = []
            for t in range((xe - xb) * n1 * n2):
                got.append((xb + t // (n1 * n2), (t // n2) % n1, t % n2))
            assert sorted(got) == list(itertools.product(range(xb, xe), range(n1), range(n2)))
            # k_return_map3 with kall: interior planes max(1, xb) <= i < min(n0 - 1, xe)
            i0, i1 = max(1, xb), min(n0 - 1, xe)
            n1i = n1 - 2
            rm = [i0 + t // (n2 * n1i) for t in range(max(i1 - i0, 0) * n1i * n2)]
            assert sorted(set(rm)) == [i for i in range(xb, xe) if 0 < i < n0 - 1]


@pytest.mark.parametrize("blocks,world", LAYOUTS)
@pytest.mark.parametrize("order", [2, 3, 4])
def test_packed_planes_are_the_neighbours_ghosts(blocks, world, order):
    g = order - 1
    plan = slabs.plan_slabs(blocks, world)
    for r, (x0, x1) in enumerate(plan):
        if r + 1 < world:   # side 1 of r feeds side 0 of r + 1
            packed = range(x1 - g, x1)
            nx0 = plan[r + 1][0]
            assert list(packed) == list(range(nx0 - g, nx0))   # what r + 1 unpacks below its slab
            assert x0 <= packed[0]                              # inside the packing slab
            assert list(range(x1, x1 + g)) == list(range(plan[r + 1][0], plan[r + 1][0] + g))


@pytest.mark.parametrize("blocks,world", LAYOUTS)
def test_every_fault_node_has_one_owner(blocks, world):
    plan = slabs.plan_slabs(blocks, world)
    nx = sum(n for _, n in blocks)

    def owners(x, blo, bxb_xe):
        return [r for r, (x0, x1) in enumerate(plan)
                if bxb_xe[r][0] <= x - blo < bxb_xe[r][1]]

    for b, (lo, n) in enumerate(blocks):
        ranges = [block_ranges([(lo, n)], x0, x1)[0][2:] for x0, x1 in plan]
        # y- or z-normal fault of this block: nodes at every x of the block
        for x in range(lo, lo + n):
            assert len(owners(x, lo, ranges)) == 1
        # x-normal fault on the block's last plane: one owner, which also updates
        # the next block's first plane
        if b + 1 < len(blocks):
            own = owners(lo + n - 1, lo, ranges)
            assert len(own) == 1
            x0, x1 = plan[own[0]]
            assert x0 <= lo + n < x1
    assert plan[-1][1] == nx
