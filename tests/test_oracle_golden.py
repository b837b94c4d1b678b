"""Oracle pins: the CPU restatement against the golden values, counts and
identities held by the reference's own test suite (test/runtests.jl)."""
import math

import numpy as np
import pytest

import oracle as orc
from diffmom_b200 import (make_rect_plate, make_icosphere, make_circular_plate, build_rwg,
                          triangle_areas, rwg_centers)


def test_analytic_1overR_centroid_golden():
    # runtests.jl:14046-14060 (Test 44): unit right triangle, centroid
    V1, V2, V3 = [0.0, 0, 0], [1.0, 0, 0], [0.0, 1, 0]
    P = np.array([1 / 3, 1 / 3, 0.0])
    S = orc.analytical_integral_1overR(P, V1, V2, V3)
    assert abs(S - 2.4072299231640093) < 1e-10


def test_analytic_1overR_offplane_golden():
    # runtests.jl:14131-14134: h = 0.5 above the centroid
    V1, V2, V3 = [0.0, 0, 0], [1.0, 0, 0], [0.0, 1, 0]
    P = np.array([1 / 3, 1 / 3, 0.5])
    S = orc.analytical_integral_1overR(P, V1, V2, V3)
    assert abs(S - 0.8515737774153572) < 1e-10


def test_analytic_1overR_properties():
    # runtests.jl:14118-14146: orientation invariance, linear scaling,
    # monotone in height, +-h symmetry
    V1, V2, V3 = np.array([0.0, 0, 0]), np.array([1.0, 0, 0]), np.array([0.0, 1, 0])
    P = (V1 + V2 + V3) / 3
    S = orc.analytical_integral_1overR(P, V1, V2, V3)
    assert abs(S - orc.analytical_integral_1overR(P, V1, V3, V2)) < 1e-12
    assert abs(orc.analytical_integral_1overR(2 * P, 2 * V1, 2 * V2, 2 * V3) - 2 * S) < 1e-10
    h = lambda z: orc.analytical_integral_1overR(P + [0, 0, z], V1, V2, V3)
    assert S > h(0.1) > h(0.5) > h(1.0) > 0
    assert abs(h(0.5) - h(-0.5)) < 1e-12
    assert math.isfinite(orc.analytical_integral_1overR(V1, V1, V2, V3))
    with pytest.raises(ValueError):
        orc.analytical_integral_1overR([math.nan, 0, 0], V1, V2, V3)
    with pytest.raises(ValueError):
        orc.analytical_integral_1overR(P + [0, 0, 0.5], V1, V1, V1)


def test_green_closed_form():
    # runtests.jl:1555-1565 (Test 2)
    k0 = 2 * math.pi / 0.1
    r1, r2 = np.zeros(3), np.array([0.05, 0, 0])
    R = 0.05
    G = orc.greens(r1, r2, k0)
    assert abs(G - np.exp(-1j * k0 * R) / (4 * math.pi * R)) < 1e-14
    assert abs(orc.greens(r1, r2, k0) - orc.greens(r2, r1, k0)) < 1e-14
    # smooth kernel: (exp(-ikR)-1)/(4 pi R), limit -ik/(4 pi) at R=0
    for R in (1e-6, 1e-3, 0.004, 0.05):
        gs = orc.greens_smooth(r1, [R, 0, 0], k0)
        ref = np.expm1(-1j * k0 * R) / (4 * math.pi * R)
        assert abs(gs - ref) <= 1e-13 * abs(ref)
    assert abs(orc.greens_smooth(r1, r1, k0) - (-1j * k0 / (4 * math.pi))) < 1e-15


def test_quadrature_rules_integrate_polynomials():
    # Quadrature.jl:17-54: degree-2 (order 3) and degree-5 (order 7) exactness
    for order, deg in ((1, 1), (3, 2), (4, 3), (7, 5)):
        xi, w = orc.tri_quad_rule(order)
        for p in range(deg + 1):
            for q in range(deg + 1 - p):
                exact = math.factorial(p) * math.factorial(q) / math.factorial(p + q + 2)
                val = float(np.sum(w * xi[:, 0] ** p * xi[:, 1] ** q))
                assert abs(val - exact) < 5e-13, (order, p, q)


def test_rect_plate_counts_and_rwg():
    # runtests.jl:487-560 (Test 1): Nv=(Nx+1)(Ny+1), Nt=2NxNy
    m = make_rect_plate(0.1, 0.1, 3, 3)
    assert m.nvertices == 16 and m.ntriangles == 18
    r = build_rwg(m)
    assert r.nedges == 3 * 9 - 6  # interior edges of a 3x3 split grid
    assert np.all(r.tplus < r.tminus)
    # config C3 size: 60x60 plate -> 10,680 RWG
    m3 = make_rect_plate(0.3, 0.3, 60, 60)
    assert m3.ntriangles == 7200 and build_rwg(m3).nedges == 3 * 3600 - 120


def test_adjacent_pair_count_4x4():
    # runtests.jl:14197-14200 (Test 45): 4x4 plate has 40 edge-adjacent pairs
    m = make_rect_plate(0.2, 0.2, 4, 4)
    r = build_rwg(m)
    c = orc.OracleCache(m, r, quad_order=4)
    assert c.adjacent_pair_count() == 40


def test_icosphere_and_circular_counts():
    s = make_icosphere(0.05, 4)
    assert s.ntriangles == 5120 and s.nvertices == 2562
    assert build_rwg(s).nedges == 7680
    d = make_circular_plate(0.1, 5, 12)
    Nt = 12 * (2 * 5 - 1)
    assert d.ntriangles == Nt and build_rwg(d).nedges == (3 * Nt - 12) // 2


def _plate_system(Nx=6, L=0.1, quad=3):
    m = make_rect_plate(L, L, Nx, Nx)
    r = build_rwg(m)
    k = 2 * math.pi / 0.1
    c = orc.OracleCache(m, r, quad_order=quad)
    return m, r, k, c


def test_assembly_symmetry_and_entry_consistency():
    m, r, k, c = _plate_system()
    Z = c.assemble_z(k)
    assert np.all(np.isfinite(Z))
    assert np.max(np.abs(Z - Z.T)) == 0.0  # canonical m<=n rule: bitwise symmetric
    idx = np.array([1, 5, 17, 60]), np.array([1, 40, 17, 2])
    e = c.entries(k, *idx)
    assert np.array_equal(e, Z[idx[0] - 1, idx[1] - 1])
    assert orc.fallback_count() == 0


def test_adjacent_quad_convergence_4x4():
    # runtests.jl:14250-14256: quad order 3 -> 4 changes Z by < 15 %
    m = make_rect_plate(0.2, 0.2, 4, 4)
    r = build_rwg(m)
    k = 2 * math.pi * 3e9 / 299792458.0
    Z3 = orc.OracleCache(m, r, 3).assemble_z(k)
    Z4 = orc.OracleCache(m, r, 4).assemble_z(k)
    assert np.max(np.abs(Z4 - Z3)) / np.max(np.abs(Z4)) < 0.15
    assert np.max(np.abs(Z4 - Z4.T)) / np.max(np.abs(Z4)) < 0.02


def test_direct_solve_residual_plate():
    # runtests.jl:2287-2310 (Test 4): ||Z I - v|| / ||v|| < 1e-10
    m, r, k, c = _plate_system()
    Z = c.assemble_z(k)
    v = c.plane_wave_rhs([0, 0, -k], 1.0, [1, 0, 0])
    I = np.linalg.solve(Z, v)
    assert np.linalg.norm(Z @ I - v) / np.linalg.norm(v) < 1e-10


def test_oracle_gmres_matches_direct_with_nearfield():
    # runtests.jl:9080-9089, 9133-9143 (Tests 19/20): NF-GMRES vs direct < 1e-6
    m, r, k, c = _plate_system(Nx=8, L=0.2)
    Z = c.assemble_z(k)
    v = c.plane_wave_rhs([0, 0, -k], 1.0, [1, 0, 0])
    I = np.linalg.solve(Z, v)
    Znf = orc.nearfield_matrix(Z, rwg_centers(m, r), 0.05)
    Minv = np.linalg.inv(Znf)
    for side in ("left", "right"):
        x, it, ok = orc.gmres(Z, v, M=Minv, side=side, rtol=1e-8, itmax=200)
        assert ok
        assert np.linalg.norm(x - I) / np.linalg.norm(I) < 1e-6


def test_mie_gate_icosphere():
    # runtests.jl:5176-5240 (Test 13): icosphere subdiv 2, r = 5 cm, 2 GHz,
    # bistatic phi cut vs Mie: MAE < 0.5 dB, RMSE < 0.6, max < 1.2, backscatter < 1.2
    from diffmom_b200.api import make_sph_grid
    mesh = make_icosphere(0.05, 2)
    rwg = build_rwg(mesh)
    f = 2.0e9
    k = 2 * math.pi * f / 299792458.0
    c = orc.OracleCache(mesh, rwg, 3)
    Z = c.assemble_z(k)
    v = c.plane_wave_rhs([0, 0, -k], 1.0, [1, 0, 0])
    I = np.linalg.solve(Z, v)
    assert np.linalg.norm(Z @ I - v) / np.linalg.norm(v) < 1e-10
    grid = make_sph_grid(37, 18)
    G = c.radiation_vectors(grid.rhat, k)
    E = (G @ I).reshape(-1, 3).T
    sig = 4 * math.pi * np.sum(np.abs(E) ** 2, axis=0)
    a = float(np.mean(np.linalg.norm(mesh.xyz - mesh.xyz.mean(axis=0), axis=1)))
    phi0 = grid.phi.min()
    cut = np.flatnonzero(np.abs(grid.phi - phi0) < 1e-12)
    cut = cut[np.argsort(grid.theta[cut])]
    mie = np.array([orc.mie_bistatic_rcs_pec(k, a, [0, 0, -1], [1, 0, 0], grid.rhat[q]) for q in cut])
    d = 10 * np.log10(np.maximum(sig[cut], 1e-30)) - 10 * np.log10(np.maximum(mie, 1e-30))
    assert np.mean(np.abs(d)) < 0.5
    assert math.sqrt(np.mean(d ** 2)) < 0.6
    assert np.max(np.abs(d)) < 1.2
    back = int(np.argmax(grid.rhat @ np.array([0, 0, 1.0])))
    sb = 4 * math.pi * np.sum(np.abs(E[:, back]) ** 2)
    mb = orc.mie_bistatic_rcs_pec(k, a, [0, 0, -1], [1, 0, 0], [0, 0, 1])
    assert abs(10 * math.log10(sb) - 10 * math.log10(mb)) < 1.2


def test_mie_large_sphere_optical_limit():
    # published Mie behaviour: backscatter of a PEC sphere tends to pi a^2
    a = 1.0
    k = 60.0
    s = orc.mie_bistatic_rcs_pec(k, a, [0, 0, -1], [1, 0, 0], [0, 0, 1])
    assert abs(s / (math.pi * a * a) - 1) < 0.1


def test_areas_match_oracle():
    m = make_icosphere(1.0, 2)
    a = triangle_areas(m)
    for t in range(0, m.ntriangles, 37):
        v = m.xyz[m.tri[t] - 1]
        ref = orc.lib().orc_triangle_area(*[orc._d(np.ascontiguousarray(v[i])) for i in range(3)])
        assert a[t] == ref


def test_golden_fixtures_reproduce():
    # the committed fixtures (tests/golden/make_golden.py) still match the oracle
    from pathlib import Path
    g = np.load(Path(__file__).parent / "golden" / "c1_plate.npz")
    m = make_rect_plate(0.1, 0.1, 6, 6)
    oc = orc.OracleCache(m, build_rwg(m), 3)
    Z = oc.assemble_z(float(g["k"]))
    assert np.array_equal(Z, g["Z"])
    assert np.linalg.norm(g["Z"] @ g["I"] - g["v"]) <= 1e-10 * np.linalg.norm(g["v"])
    assert np.all(g["sigma_cut"] > 0) and np.all(g["sigma_mono"] > 0)
