"""Cluster tree, admissibility and block tasks of the H-matrix operator: the
library's host code (dmb_aca_plan / dmb_aca_admissible, no GPU) against the
oracle's restatement of src/fast/ClusterTree.jl and src/fast/ACA.jl:696-738,
and the oracle itself against facts the reference's tests state."""
import math

import numpy as np
import pytest

from diffmom_b200 import (make_rect_plate, make_circular_plate, build_rwg, rwg_centers, build_cluster_tree,
                          aca_block_tasks, is_admissible, leaf_nodes, cluster_diameter, cluster_distance)
from diffmom_b200 import _native as nat

import aca_oracle as ao


def _plate_centers(nx, ny, a=1.0, b=1.0):
    m = make_rect_plate(a, b, nx, ny)
    return rwg_centers(m, build_rwg(m))


def _compare(centers, leaf, eta):
    tree = build_cluster_tree(centers, leaf)
    otree = ao.build_cluster_tree(centers, leaf)
    np.testing.assert_array_equal(tree.perm - 1, otree.perm)
    assert len(tree.nodes) == len(otree.nodes)
    for nd, on in zip(tree.nodes, otree.nodes):
        assert (nd.indices.start - 1, nd.indices.stop - 2) == (on.lo, on.hi)
        assert (nd.left - 1, nd.right - 1, nd.level) == (on.left, on.right, on.level)
        assert tuple(nd.bbox_min) == on.bmin and tuple(nd.bbox_max) == on.bmax
    tasks = aca_block_tasks(centers, leaf, eta)
    otasks = ao.enum_block_tasks(otree, eta)
    assert [(r - 1, c - 1, 1 if k == "lowrank" else 0) for r, c, k in tasks] == otasks
    return tree, otasks


def test_oracle_pins_reference_scale_fixture():
    # the reference's scale-invariance test: make_rect_plate(1.0, 1.0, 1, 2)
    # with leaf_size=1, eta=1.5 has four admissible far blocks, each of rank
    # at most one (three collinear centres: two 1x1 blocks between the leaves
    # of the two-point cluster, and that cluster against the third point)
    c = _plate_centers(1, 2)
    assert c.shape[0] == 3
    tree = ao.build_cluster_tree(c, 1)
    tasks = ao.enum_block_tasks(tree, 1.5)
    far = [t for t in tasks if t[2] == 1]
    assert len(far) == 4
    shapes = sorted((tree.nodes[rn].hi - tree.nodes[rn].lo + 1, tree.nodes[cn].hi - tree.nodes[cn].lo + 1)
                    for rn, cn, _ in far)
    assert shapes == [(1, 1), (1, 1), (1, 2), (2, 1)]
    # every ordered pair of unknowns lies in exactly one block
    cover = np.zeros((3, 3), int)
    for rn, cn, _ in tasks:
        r, cc = tree.nodes[rn], tree.nodes[cn]
        cover[r.lo:r.hi + 1, cc.lo:cc.hi + 1] += 1
    assert np.all(cover == 1)


@pytest.mark.parametrize("leaf,eta", [(1, 1.5), (4, 1.0), (8, 1.5), (64, 1.5), (16, 0.8)])
def test_plan_matches_oracle_on_plates(leaf, eta):
    # regular plates: many equal coordinates, so the stable median split and
    # boundary-exact admissibility both matter
    for nx, ny in ((6, 6), (20, 20), (24, 7)):
        c = _plate_centers(nx, ny)
        _compare(c, leaf, eta)


def test_plan_matches_oracle_on_curved_and_random_points():
    m = make_circular_plate(0.5, 8, 24)
    _compare(rwg_centers(m, build_rwg(m)), 8, 1.5)
    rng = np.random.default_rng(7)
    pts = rng.standard_normal((700, 3))
    pts[::7, 2] = 0.0
    pts[1::7, 2] = -0.0
    _compare(pts, 16, 1.5)
    _compare(pts, 3, 2.0)


def test_tasks_tile_the_matrix():
    c = _plate_centers(12, 10)
    tree, tasks = _compare(c, 8, 1.5)
    N = c.shape[0]
    cover = np.zeros((N, N), np.int8)
    for rn, cn, _ in tasks:
        r, cc = tree.nodes[rn], tree.nodes[cn]
        cover[r.indices.start - 1:r.indices.stop - 1, cc.indices.start - 1:cc.indices.stop - 1] += 1
    assert np.all(cover == 1)
    # dense blocks pair leaves; the diagonal blocks are never admissible
    leaves = set(leaf_nodes(tree))
    for rn, cn, kind in tasks:
        if kind == 0:
            assert rn + 1 in leaves and cn + 1 in leaves
        if rn == cn:
            assert kind == 0


def _box(lo, hi):
    return ao.Node(0, 0, tuple(lo), tuple(hi))


def test_admissibility_exact_on_the_boundary():
    lib = nat.load_library()

    def lib_adm(a, b, eta):
        out = nat.ctypes.c_int()
        bi = np.array(a.bmin + a.bmax, dtype=np.float64)
        bj = np.array(b.bmin + b.bmax, dtype=np.float64)
        nat.check_free(lib, lib.dmb_aca_admissible(nat.dptr(bi), nat.dptr(bj), eta, nat.ctypes.byref(out)))
        return bool(out.value)

    cases = []
    # diameter 0.3 (in units that are not binary fractions) and gap exactly
    # 0.2: 0.3 <= 1.5 * 0.2 sits on the boundary in exact arithmetic of the
    # stored doubles or one ulp beside it
    for x0 in (0.0, 0.1, 1e-3, 7.0):
        for d in (0.3, 0.1 * 3, 3.0, 0.7):
            for g in (d / 1.5, math.nextafter(d / 1.5, 0), math.nextafter(d / 1.5, 1)):
                a = _box((x0, 0.0, 0.0), (x0 + d, d / 2, 0.0))
                b = _box((x0 + d + g, 0.0, 0.0), (x0 + 2 * d + g, d, 0.0))
                cases.append((a, b, 1.5))
    # diagonal gaps: |gap| = sqrt(gx^2 + gy^2)
    for gx, gy in ((0.3, 0.4), (3.0, 4.0), (0.1, 0.2)):
        a = _box((0.0, 0.0, 0.0), (0.75, 0.75, 0.0))
        b = _box((0.75 + gx, 0.75 + gy, 0.0), (1.5 + gx, 1.5 + gy, 0.0))
        cases.append((a, b, 0.75 / math.hypot(gx, gy)))
        cases.append((a, b, math.nextafter(0.75 / math.hypot(gx, gy), 0)))
    seen = set()
    for a, b, eta in cases:
        o = ao.box_admissible(a, b, eta)
        assert lib_adm(a, b, eta) == o
        assert lib_adm(b, a, eta) == ao.box_admissible(b, a, eta)
        seen.add(o)
    assert seen == {True, False}


def test_plan_errors():
    c = _plate_centers(2, 2)
    with pytest.raises(ValueError, match="leaf_size"):
        build_cluster_tree(c, 0)
    with pytest.raises(ValueError, match="eta"):
        aca_block_tasks(c, 1, float("nan"))
    with pytest.raises(ValueError, match="eta"):
        aca_block_tasks(c, 1, 0.0)
    with pytest.raises(ValueError, match="max_block_tasks"):
        aca_block_tasks(c, 1, 1.5, max_block_tasks=1)
    with pytest.raises(ValueError, match="empty"):
        build_cluster_tree(np.zeros((0, 3)), 4)
    bad = c.copy()
    bad[2, 1] = np.inf
    with pytest.raises(ValueError, match="finite"):
        build_cluster_tree(bad, 4)


def test_tree_helpers():
    c = _plate_centers(10, 10)
    tree = build_cluster_tree(c, 8)
    leaves = leaf_nodes(tree)
    assert sum(len(tree.nodes[i - 1].indices) for i in leaves) == c.shape[0]
    np.testing.assert_array_equal(tree.iperm[tree.perm - 1], np.arange(1, c.shape[0] + 1))
    ot = ao.build_cluster_tree(c, 8)
    for i in (1, 2, leaves[0], leaves[-1]):
        assert cluster_diameter(tree, i) == ao.cluster_diameter(ot, i - 1)
    for i, j in ((leaves[0], leaves[-1]), (leaves[1], leaves[5]), (2, 3)):
        assert is_admissible(tree, i, j, 1.5) == ao.is_admissible(ot, i - 1, j - 1, 1.5)
        assert cluster_distance(tree, i, j) >= 0


def test_oracle_aca_and_product_on_a_smooth_kernel():
    # two separated point clouds: exp(-i k r) / r between them is numerically
    # low rank, the oracle's ACA meets its relative tolerance, and the
    # H-matrix product of oracle blocks equals the dense product
    rng = np.random.default_rng(3)
    x = rng.uniform(0, 1, (60, 3))
    y = rng.uniform(0, 1, (50, 3)) + np.array([4.0, 0, 0])
    r = np.linalg.norm(x[:, None] - y[None], axis=2)
    B = np.exp(-2j * r) / r
    for tol in (1e-4, 1e-8):
        U, V, conv = ao.aca_lowrank(B, tol, 50)
        assert conv and U.shape[1] < 50
        assert np.linalg.norm(U @ V.conj().T - B) <= 10 * tol * np.linalg.norm(B)
    pts = np.vstack([x, y])
    rr = np.linalg.norm(pts[:, None] - pts[None], axis=2) + np.eye(110)
    Z = np.exp(-2j * rr) / rr
    tree, tasks, blocks = ao.build_hmatrix(Z, pts, leaf_size=8, eta=1.5, aca_tol=1e-10, max_rank=40)
    assert any(b.kind == 1 for b in blocks)
    v = rng.standard_normal(110) + 1j * rng.standard_normal(110)
    for mode, A in ((0, Z), (1, Z.conj().T), (2, Z.T)):
        y_h = ao.hmatrix_matvec(blocks, tree.perm, v, mode)
        assert np.linalg.norm(y_h - A @ v) <= 1e-8 * np.linalg.norm(A @ v)


def test_operator_arguments_rejected_before_any_device_work():
    # build_aca_operator / aca_lowrank validate like ACA.jl:332-340 and
    # :802-850 before a device context exists
    from diffmom_b200 import build_aca_operator, aca_lowrank, EFIECache
    m = make_rect_plate(1.0, 1.0, 2, 2)
    r = build_rwg(m)
    for kw in ({"aca_tol": math.inf}, {"aca_tol": 0.0}, {"aca_tol": math.nan}, {"max_rank": 0},
               {"leaf_size": 0}, {"eta": math.nan}, {"eta": 0.0}, {"max_block_tasks": 0},
               {"max_storage_bytes": 0}, {"max_green_cache_bytes": 0}, {"max_green_cache_entries": -1},
               {"max_adjacency_pairs": 0}, {"max_cache_bytes": 1}, {"quad_order": 5},
               {"quad_order": 3, "max_green_cache_bytes": 16 * 9 - 1}):
        with pytest.raises(ValueError):
            build_aca_operator(m, r, 2 * math.pi, **kw)
    other = build_rwg(make_rect_plate(1.0, 1.0, 2, 2))
    with pytest.raises(ValueError, match="different mesh"):
        build_aca_operator(m, other, 2 * math.pi)
    cache = EFIECache(device=None, k=2 * math.pi)
    for kw in ({"tol": 0.0}, {"tol": math.inf}, {"tol": math.nan}, {"max_rank": 0}, {"max_rank": -1}):
        with pytest.raises(ValueError):
            aca_lowrank(cache, [1], [1], **kw)


def test_scaled_product_contract():
    # mul!(y, A, x, alpha, beta) semantics of the Python operator wrapper
    from diffmom_b200.aca import _scaled
    Ax = np.array([1 + 2j, -3.0, 0.5j])
    np.testing.assert_array_equal(_scaled(Ax, 1.0, 0.0, None), Ax)
    y = np.array([np.nan, 1.0, 2.0], dtype=complex)  # beta = 0 ignores y
    np.testing.assert_array_equal(_scaled(Ax, 2.0, 0.0, y), 2.0 * Ax)
    y = np.array([1.0, 1.0, 1.0], dtype=complex)
    np.testing.assert_allclose(_scaled(Ax, 0.5 - 1j, 2.0, y), (0.5 - 1j) * Ax + 2.0)
    with pytest.raises(OverflowError):
        _scaled(np.array([1e308 + 0j]), 10.0, 0.0, np.zeros(1, complex))


def test_plan_abi_two_call_protocol_and_task_limit():
    # dmb_aca_plan: the task count always comes back; the task array is
    # written only when its capacity suffices; max_block_tasks equal to the
    # task count passes, one less fails
    import ctypes
    lib = nat.load_library()
    c = np.ascontiguousarray(_plate_centers(8, 8))
    n = c.shape[0]
    perm = np.empty(n, np.int64)
    nn, nt = ctypes.c_int64(), ctypes.c_int64()
    nat.check_free(lib, lib.dmb_aca_plan(nat.dptr(c), n, 4, 1.5, 1 << 40, nat.lptr(perm), ctypes.byref(nn), None,
                                         None, ctypes.byref(nt), None, 0))
    count = nt.value
    assert count > 1 and sorted(perm.tolist()) == list(range(1, n + 1))
    small = np.full((count - 1, 5), -7, np.int64)
    nat.check_free(lib, lib.dmb_aca_plan(nat.dptr(c), n, 4, 1.5, 1 << 40, None, None, None, None,
                                         ctypes.byref(nt), nat.lptr(small), count - 1))
    assert nt.value == count and np.all(small == -7)
    full = np.empty((count, 5), np.int64)
    nat.check_free(lib, lib.dmb_aca_plan(nat.dptr(c), n, 4, 1.5, count, None, None, None, None,
                                         ctypes.byref(nt), nat.lptr(full), count))
    assert set(full[:, 2].tolist()) <= {0, 1} and np.all(full[:, :2] >= 1)
    with pytest.raises(ValueError, match="max_block_tasks"):
        nat.check_free(lib, lib.dmb_aca_plan(nat.dptr(c), n, 4, 1.5, count - 1, None, None, None, None,
                                             ctypes.byref(nt), None, 0))


def test_reference_cluster_tree_fixtures():
    # runtests.jl:9318-9395: resource bounds, invalid centres, tree invariants
    # and the rounded-boundary admissibility pair
    from diffmom_b200.aca import cluster_tree_resource_bounds, ClusterTree, ClusterNode
    c = _plate_centers(12, 12)
    N = c.shape[0]
    tree = build_cluster_tree(c, 8)
    nb, sb = cluster_tree_resource_bounds(N, 8)
    with pytest.raises(ValueError, match="max_nodes"):
        build_cluster_tree(c, 8, max_nodes=nb - 1)
    with pytest.raises(ValueError, match="max_storage_bytes"):
        build_cluster_tree(c, 8, max_nodes=nb, max_storage_bytes=sb - 1)
    np.testing.assert_array_equal(build_cluster_tree(c, 8, max_nodes=nb, max_storage_bytes=sb).perm, tree.perm)
    for bad in ([[math.nan, 0.0, 0.0]], [[-np.finfo(float).max, 0, 0], [np.finfo(float).max, 0, 0]]):
        with pytest.raises(ValueError):
            build_cluster_tree(np.array(bad, dtype=float), 8)
    assert sorted(tree.perm.tolist()) == list(range(1, N + 1))
    np.testing.assert_array_equal(tree.iperm[tree.perm - 1], np.arange(1, N + 1))
    assert tree.nodes[0].indices == range(1, N + 1)
    for i in leaf_nodes(tree):
        assert len(tree.nodes[i - 1].indices) <= 8
    assert not is_admissible(tree, leaf_nodes(tree)[0], leaf_nodes(tree)[0])
    for eta in (math.nan, 0.0):
        with pytest.raises(ValueError):
            is_admissible(tree, 1, 1, eta=eta)
    # the stored boxes sit exactly 1.0 apart after rounding, and the exact
    # decision separates them: prevfloat(2^-26) stays dense, 2^-26 is admissible
    bx = math.nextafter(1.0, 0.0)

    def pair(y):
        nodes = [ClusterNode(range(1, 2), np.array([0.0, 0.0, 0.0]), np.array([0.0, 0.0, 1.0]), 0, 0, 0),
                 ClusterNode(range(2, 3), np.array([bx, y, 0.0]), np.array([bx, y, 1.0]), 0, 0, 0)]
        return ClusterTree(nodes, np.array([1, 2]), np.array([1, 2]), 1)
    inside, outside = pair(math.nextafter(2.0 ** -26, 0.0)), pair(2.0 ** -26)
    assert cluster_distance(inside, 1, 2) == 1.0 and cluster_distance(outside, 1, 2) == 1.0
    assert not is_admissible(inside, 1, 2, eta=1.0)
    assert is_admissible(outside, 1, 2, eta=1.0)
    # and the oracle's exact rationals agree
    assert not ao.box_admissible(ao.Node(0, 0, tuple(inside.nodes[0].bbox_min), tuple(inside.nodes[0].bbox_max)),
                                 ao.Node(0, 0, tuple(inside.nodes[1].bbox_min), tuple(inside.nodes[1].bbox_max)), 1.0)
    assert ao.box_admissible(ao.Node(0, 0, tuple(outside.nodes[0].bbox_min), tuple(outside.nodes[0].bbox_max)),
                             ao.Node(0, 0, tuple(outside.nodes[1].bbox_min), tuple(outside.nodes[1].bbox_max)), 1.0)


def test_oracle_stopping_rule_is_scale_invariant():
    # runtests.jl:9456-9500 on the oracle: the relative Frobenius rule in
    # scaled magnitudes gives the same rank and the same factors (up to the
    # scale) at 1e-200 and 1e200, where squared norms would under/overflow
    rng = np.random.default_rng(11)
    x = rng.uniform(0, 1, (40, 3))
    y = rng.uniform(0, 1, (30, 3)) + np.array([3.0, 0.5, 0])
    r = np.linalg.norm(x[:, None] - y[None], axis=2)
    B = np.exp(-3j * r) / r
    U0, V0, conv0 = ao.aca_lowrank(B, 1e-3, 20)
    assert conv0 and U0.shape[1] < 20
    ref = U0 @ V0.conj().T
    for scale in (1e-200, 1e200):
        U, V, conv = ao.aca_lowrank(B * scale, 1e-3, 20)
        assert conv == conv0 and U.shape[1] == U0.shape[1]
        np.testing.assert_allclose((U @ V.conj().T) / scale, ref, rtol=5e-13, atol=0)


def test_solve_scattering_aca_arguments_rejected_on_the_host():
    from diffmom_b200 import solve_scattering, make_plane_wave
    m = make_rect_plate(0.1, 0.1, 2, 2)
    k = 2 * math.pi * 3e9 / 299792458.0
    pw = make_plane_wave(np.array([0.0, 0.0, -k]), 1.0, np.array([1.0, 0.0, 0.0]))
    with pytest.raises(ValueError, match="surface_impedance"):
        solve_scattering(m, 3e9, pw, method="aca_gmres", surface_impedance=np.ones(m.ntriangles))
    with pytest.raises(ValueError, match="method"):
        solve_scattering(m, 3e9, pw, method="mlfma")


def test_oracle_hmatrix_on_an_efie_matrix():
    # the oracle's build_aca_operator restatement on the oracle's own EFIE Z
    # (plate of 1.5 wavelengths at 3 GHz): the product meets the tolerance,
    # and a looser tolerance never raises a block's rank
    import oracle as orc
    m = make_rect_plate(0.15, 0.15, 10, 10)
    r = build_rwg(m)
    k = 2 * math.pi * 3e9 / 299792458.0
    Z = orc.OracleCache(m, r, 3).assemble_z(k)
    c = rwg_centers(m, r)
    x = np.random.default_rng(2).standard_normal(r.nedges) + 0j
    ranks = {}
    for tol in (1e-8, 1e-4):
        tree, tasks, blocks = ao.build_hmatrix(Z, c, leaf_size=16, eta=1.5, aca_tol=tol, max_rank=50)
        lr = [b for b in blocks if b.kind == 1]
        # (the far blocks of so small a plate are near full rank: compression
        # shows at larger N, as the GPU tests on the 10,680-RWG plate check)
        assert lr
        y = ao.hmatrix_matvec(blocks, tree.perm, x, 0)
        err = np.linalg.norm(y - Z @ x) / np.linalg.norm(Z @ x)
        assert err < 100 * tol
        ranks[tol] = [b.U.shape[1] for b in lr]
    assert all(a >= b for a, b in zip(ranks[1e-8], ranks[1e-4]))


def test_plan_matches_committed_fixture():
    # tests/golden/aca_plan_plate.npz (written by tests/golden/make_golden.py
    # from the oracle): the library's plan, bit for bit
    from pathlib import Path
    g = np.load(Path(__file__).resolve().parent / "golden" / "aca_plan_plate.npz")
    c = g["centers"]
    for leaf in (4, 16):
        tree = build_cluster_tree(c, leaf)
        np.testing.assert_array_equal(tree.perm - 1, g[f"perm_{leaf}"])
        nodes = np.array([[n.indices.start - 1, n.indices.stop - 2, n.left - 1, n.right - 1, n.level]
                          for n in tree.nodes])
        np.testing.assert_array_equal(nodes, g[f"nodes_{leaf}"])
        boxes = np.array([np.concatenate([n.bbox_min, n.bbox_max]) for n in tree.nodes])
        np.testing.assert_array_equal(boxes, g[f"boxes_{leaf}"])
        tasks = np.array([(r - 1, cc - 1, 1 if k == "lowrank" else 0) for r, cc, k in aca_block_tasks(c, leaf, 1.5)])
        np.testing.assert_array_equal(tasks, g[f"tasks_{leaf}"])
