"""Host logic of the batched multi-block form: halo-map generators and checks.

The gather semantics (dst <- stage input or stage output at src) are
simulated with numpy on padded arrays; the single-block periodic rule is
restated here with scalar loops, independently of the vectorised generators.
"""
import itertools

import numpy as np
import pytest

from chimera_comp_les_b200 import batch as B


def bc_source_scalar(i, j, k, M):
    """FormBCS (rhs.c:1107-1227) + DMGlobalToLocal for one non-interior node of
    a fully periodic block: (si, sj, sk, from_stage_input)."""
    mx, my, mz = M
    w = lambda x, m: x + m if x < 0 else (x - m if x >= m else x)
    oi, oj, ok = w(i, mx), w(j, my), w(k, mz)
    if 0 < oi < mx - 1 and 0 < oj < my - 1 and 0 < ok < mz - 1:
        return oi, oj, ok, 0
    if ok == 0:
        return oi, oj, -2, 1
    if ok == mz - 1:
        return oi, oj, mz + 1, 1
    if oj == 0:
        return oi, -2, ok, 1
    if oj == my - 1:
        return oi, my + 1, ok, 1
    if oi == 0:
        return -2, oj, ok, 1
    return mx + 1, oj, ok, 1


def interior(d, i, j, k):
    return 1 <= i <= d[0] - 2 and 1 <= j <= d[1] - 2 and 1 <= k <= d[2] - 2


def padded(d, rng):
    return rng.standard_normal((d[2] + 4, d[1] + 4, d[0] + 4))


def at(a, i, j, k):
    return a[k + 2, j + 2, i + 2]


def global_stage(M, qin, qout):
    res = qout.copy()
    for k, j, i in itertools.product(range(-2, M[2] + 2), range(-2, M[1] + 2), range(-2, M[0] + 2)):
        if interior(M, i, j, k):
            continue
        si, sj, sk, fin = bc_source_scalar(i, j, k, M)
        res[k + 2, j + 2, i + 2] = at(qin if fin else qout, si, sj, sk)
    return res


def apply_map(entries, arrs_in, arrs_out):
    res = [a.copy() for a in arrs_out]
    for r in entries:
        src = arrs_in[r[4]] if r[8] else arrs_out[r[4]]
        res[r[0]][r[3] + 2, r[2] + 2, r[1] + 2] = src[r[7] + 2, r[6] + 2, r[5] + 2]
    return res


def block_slice(g, off, d):
    return g[off[2]:off[2] + d[2] + 4, off[1]:off[1] + d[1] + 4, off[0]:off[0] + d[0] + 4].copy()


def test_self_periodic_matches_scalar_rule():
    dims = [(7, 6, 8), (9, 7, 6)]
    st, wr = B.halo_maps_self_periodic(dims)
    for r in st:
        d = dims[r[0]]
        assert r[0] == r[4]
        assert tuple(r[5:9]) == bc_source_scalar(r[1], r[2], r[3], d)
    # every non-interior node exactly once
    for b, d in enumerate(dims):
        n_non = (d[0] + 4) * (d[1] + 4) * (d[2] + 4) - (d[0] - 2) * (d[1] - 2) * (d[2] - 2)
        assert (st[:, 0] == b).sum() == n_non
    B.check_halo_map(dims, st, B.HALO_STAGE)
    B.check_halo_map(dims, wr, B.HALO_WRAP)


def test_self_periodic_skips_coded_blocks():
    """Blocks with face codes run their own FormBCS: the generator leaves them
    out and keeps every other block's entries unchanged."""
    dims = [(7, 6, 8), (9, 7, 6), (8, 8, 7)]
    st, wr = B.halo_maps_self_periodic(dims)
    st1, wr1 = B.halo_maps_self_periodic(dims, coded=[1])
    assert not (st1[:, 0] == 1).any() and not (wr1[:, 0] == 1).any()
    assert np.array_equal(st1, st[st[:, 0] != 1]) and np.array_equal(wr1, wr[wr[:, 0] != 1])


def test_decomposed_single_part_equals_self_periodic():
    M = (9, 8, 10)
    parts = B.decompose(M, [[7], [6], [8]])
    st, wr = B.halo_maps_decomposed(M, parts)
    st0, wr0 = B.halo_maps_self_periodic([M])
    key = lambda a: sorted(map(tuple, a.tolist()))
    assert key(st) == key(st0)
    assert key(wr) == key(wr0)


@pytest.mark.parametrize("cuts", [([5, 7], [10], [4, 6, 5]), ([12], [4, 6], [15]), ([4, 4, 4], [5, 5], [7, 8])])
def test_decomposed_stage_map_reproduces_undivided_box(cuts):
    M = (sum(cuts[0]) + 2, sum(cuts[1]) + 2, sum(cuts[2]) + 2)
    rng = np.random.default_rng(7)
    qin, qout = padded(M, rng), padded(M, rng)
    want = global_stage(M, qin, qout)
    parts = B.decompose(M, cuts)
    st, wr = B.halo_maps_decomposed(M, parts)
    dims = [p[1] for p in parts]
    B.check_halo_map(dims, st, B.HALO_STAGE)
    B.check_halo_map(dims, wr, B.HALO_WRAP)
    ins, outs = [], []
    for off, d in parts:
        ins.append(block_slice(qin, off, d))
        o = block_slice(qout, off, d)
        # non-interior nodes of the stage output are not written by the stage:
        # the gather must not read them
        mask = np.ones_like(o, dtype=bool)
        mask[3:d[2] + 1, 3:d[1] + 1, 3:d[0] + 1] = False
        o[mask] = np.nan
        outs.append(o)
    got = apply_map(st, ins, outs)
    for (off, d), g in zip(parts, got):
        np.testing.assert_array_equal(g, block_slice(want, off, d))


def test_decomposed_wrap_map_reproduces_ghost_fill():
    cuts = ([5, 6], [8], [4, 5, 6])
    M = (sum(cuts[0]) + 2, sum(cuts[1]) + 2, sum(cuts[2]) + 2)
    rng = np.random.default_rng(3)
    g = padded(M, rng)
    # global ghost fill: ghosts take their owned image
    want = g.copy()
    for k, j, i in itertools.product(range(-2, M[2] + 2), range(-2, M[1] + 2), range(-2, M[0] + 2)):
        w = lambda x, m: x + m if x < 0 else (x - m if x >= m else x)
        want[k + 2, j + 2, i + 2] = at(g, w(i, M[0]), w(j, M[1]), w(k, M[2]))
    parts = B.decompose(M, cuts)
    _, wr = B.halo_maps_decomposed(M, parts)
    arrs = []
    for off, d in parts:
        a = block_slice(want, off, d)
        # what a block holds before the gather: its own owned nodes, ghosts unknown,
        # and (eddy viscosity) zeros at boundary nodes that are another block's interior
        for k, j, i in itertools.product(range(-2, d[2] + 2), range(-2, d[1] + 2), range(-2, d[0] + 2)):
            own = 0 <= i < d[0] and 0 <= j < d[1] and 0 <= k < d[2]
            if not own:
                a[k + 2, j + 2, i + 2] = np.nan
            elif not interior(d, i, j, k):
                gi, gj, gk = i + off[0], j + off[1], k + off[2]
                if interior(M, gi, gj, gk):
                    a[k + 2, j + 2, i + 2] = np.nan
        arrs.append(a)
    got = apply_map(wr, arrs, arrs)
    for (off, d), a in zip(parts, got):
        np.testing.assert_array_equal(a, block_slice(want, off, d))


def test_donor_map_sources_are_donor_interior():
    rng = np.random.default_rng(11)
    dims = [tuple(int(x) for x in rng.integers(6, 14, size=3)) for _ in range(5)]
    perm = [3, 0, 4, 1, 2]
    st, wr = B.halo_maps_donor(dims, perm)
    B.check_halo_map(dims, st, B.HALO_STAGE)
    B.check_halo_map(dims, wr, B.HALO_WRAP)
    assert (st[:, 4] == np.array(perm)[st[:, 0]]).all()
    for b, d in enumerate(dims):
        n_non = (d[0] + 4) * (d[1] + 4) * (d[2] + 4) - (d[0] - 2) * (d[1] - 2) * (d[2] - 2)
        assert (st[:, 0] == b).sum() == n_non
    # a node one below the low x face reads the donor's last interior node
    r = st[(st[:, 0] == 0) & (st[:, 1] == 0) & (st[:, 2] == 3) & (st[:, 3] == 3)][0]
    assert r[5] == dims[perm[0]][0] - 2


@pytest.mark.parametrize("mistake", ["interior_dst", "duplicate", "outside", "stage_out_not_interior", "wrap_chain"])
def test_check_halo_map_rejects_planted_mistakes(mistake):
    dims = [(8, 7, 9)]
    st, wr = B.halo_maps_self_periodic(dims)
    kind = B.HALO_STAGE
    e = st.copy()
    if mistake == "interior_dst":
        e[0, 1:4] = (3, 3, 3)
    elif mistake == "duplicate":
        e[1, :4] = e[0, :4]
    elif mistake == "outside":
        e[0, 5] = dims[0][0] + 2
    elif mistake == "stage_out_not_interior":
        i = np.nonzero(e[:, 8] == 0)[0][0]
        e[i, 5:8] = (0, 0, 0)
    else:
        kind = B.HALO_WRAP
        e = wr.copy()
        e[0, 5:8] = e[1, 1:4]
    with pytest.raises(ValueError):
        B.check_halo_map(dims, e, kind)


def test_decompose_rejects_bad_cuts():
    with pytest.raises(ValueError):
        B.decompose((10, 10, 10), [[8], [4, 3], [8]])
    with pytest.raises(ValueError):
        B.decompose((10, 10, 10), [[8], [5, 3], [8]])
