"""Adjoint solves (solve_gmres_adjoint, NearFieldAdjointOperator) against the
oracle's dense Z^H, following the reference's own checks (runtests.jl
7428-7440 and 9101-9151)."""
import math

import numpy as np
import pytest

import oracle as orc
from diffmom_b200 import (EFIEDevice, NearFieldAdjointOperator, NearFieldOperator, build_rwg, make_rect_plate,
                          solve_gmres_adjoint)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def plate():
    m = make_rect_plate(0.1, 0.1, 6, 6)
    rwg = build_rwg(m)
    k = 2 * math.pi / 0.1
    Z = orc.OracleCache(m, rwg, 3).assemble_z(k)
    dev = EFIEDevice(m, rwg)
    dev.assemble(k)
    yield dev, Z, k
    dev.close()


def test_nearfield_adjoint_consistency(plate):
    dev, Z, k = plate
    P = dev.build_nearfield(0.05, "lu")
    M, Ma = NearFieldOperator(P), NearFieldAdjointOperator(P)
    rng = np.random.default_rng(3)
    x = rng.standard_normal(dev.N) + 1j * rng.standard_normal(dev.N)
    y = rng.standard_normal(dev.N) + 1j * rng.standard_normal(dev.N)
    lhs = np.vdot(M @ x, y)
    rhs = np.vdot(x, Ma @ y)
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


@pytest.mark.parametrize("pc,side", [(None, "left"), ("lu", "left"), ("lu", "right"), ("diag", "left")])
def test_adjoint_gmres_matches_dense(plate, pc, side):
    dev, Z, k = plate
    rng = np.random.default_rng(5)
    b = rng.standard_normal(dev.N) + 1j * rng.standard_normal(dev.N)
    lam_ref = np.linalg.solve(Z.conj().T, b)
    P = None if pc is None else dev.build_nearfield(0.05, pc)
    lam, st = solve_gmres_adjoint(dev, b, preconditioner=P, precond_side=side, tol=1e-10, maxiter=500)
    lam = np.asarray(lam).reshape(-1)
    assert st.solved
    assert np.linalg.norm(lam - lam_ref) <= 1e-6 * np.linalg.norm(lam_ref)


def test_adjoint_rejects_sparse_local_rows(plate):
    dev, Z, k = plate
    P = dev.build_local(0.02)
    with pytest.raises(ValueError):
        solve_gmres_adjoint(dev, np.ones(dev.N, dtype=complex), preconditioner=P)
