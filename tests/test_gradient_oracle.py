"""Impedance gradient on the CPU: the oracle's gradient_impedance
(Adjoint.jl:1081-1119) against central finite differences of
J(theta) = Re(I^H Q I), Z(theta) = Z_efie - sum_p theta_p M_p (resistive) or
- sum_p i theta_p M_p (reactive), I = Z^-1 v, lambda = Z^-H Q I -- the check the
reference's optimisation verification performs (Verification.jl)."""
import math

import numpy as np
import pytest

import oracle as orc
from diffmom_b200 import PatchPartition, build_rwg, make_rect_plate


def _quadrant_patches(mesh):
    c = mesh.xyz[mesh.tri - 1].mean(axis=1)
    return (c[:, 0] > 0).astype(int) + 2 * (c[:, 1] > 0).astype(int)


@pytest.mark.parametrize("reactive", [False, True])
def test_gradient_matches_finite_differences(reactive):
    m = make_rect_plate(0.1, 0.1, 6, 6)
    rwg = build_rwg(m)
    oc = orc.OracleCache(m, rwg, 3)
    k = 2 * math.pi / 0.1
    Ze = oc.assemble_z(k)
    v = oc.plane_wave_rhs([0, 0, -k], 1.0, [1, 0, 0])
    tp = _quadrant_patches(m)
    P = 4
    PatchPartition(tp + 1, P)  # the partition is valid for the reference type
    rng = np.random.default_rng(3)
    theta = rng.uniform(50, 200, P)
    N = Ze.shape[0]
    A = rng.standard_normal((6, N)) + 1j * rng.standard_normal((6, N))
    Q = A.conj().T @ A  # Hermitian, positive semidefinite

    def system(th):
        zs = th[tp] * (1j if reactive else 1.0)
        return oc.apply_impedance(Ze, zs)

    def J(th):
        I = np.linalg.solve(system(th), v)
        return float(np.real(I.conj() @ Q @ I))

    Z = system(theta)
    I = np.linalg.solve(Z, v)
    lam = np.linalg.solve(Z.conj().T, Q @ I)
    g = oc.gradient_impedance(I, lam, tp, P, reactive=reactive)
    for p in range(P):
        h = 1e-4 * theta[p]
        e = np.zeros(P)
        e[p] = h
        fd = (J(theta + e) - J(theta - e)) / (2 * h)
        assert abs(fd - g[p]) <= 1e-6 * max(abs(g).max(), 1e-300)


def test_columns_are_independent():
    m = make_rect_plate(0.1, 0.1, 4, 4)
    rwg = build_rwg(m)
    oc = orc.OracleCache(m, rwg, 3)
    rng = np.random.default_rng(1)
    N = rwg.nedges
    I = rng.standard_normal((N, 3)) + 1j * rng.standard_normal((N, 3))
    L = rng.standard_normal((N, 3)) + 1j * rng.standard_normal((N, 3))
    tp = np.arange(m.ntriangles) % 5
    G = oc.gradient_impedance(I, L, tp, 5)
    for r in range(3):
        np.testing.assert_allclose(G[:, r], oc.gradient_impedance(I[:, r], L[:, r], tp, 5), rtol=1e-14, atol=0)
