"""Impedance gradients on the device (dmb_gradient_impedance) against the
oracle's gradient_impedance (Adjoint.jl:1081-1119), and the device
forward / adjoint / gradient chain against the oracle's dense one."""
import math

import numpy as np
import pytest

import oracle as orc
from diffmom_b200 import (EFIEDevice, PatchPartition, build_rwg, gradient_impedance, make_rect_plate,
                          precompute_patch_mass, solve_adjoint_rhs)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def plate():
    m = make_rect_plate(0.1, 0.1, 6, 6)
    rwg = build_rwg(m)
    dev = EFIEDevice(m, rwg)
    yield m, rwg, dev, orc.OracleCache(m, rwg, 3)
    dev.close()


def _quadrants(m):
    c = m.xyz[m.tri - 1].mean(axis=1)
    return (c[:, 0] > 0).astype(int) + 2 * (c[:, 1] > 0).astype(int)


@pytest.mark.parametrize("reactive", [False, True])
@pytest.mark.parametrize("layout", ["quadrants", "per_triangle", "single"])
def test_gradient_matches_oracle(plate, reactive, layout):
    m, rwg, dev, oc = plate
    nt = m.ntriangles
    tp = {"quadrants": _quadrants(m), "per_triangle": np.arange(nt), "single": np.zeros(nt, int)}[layout]
    P = int(tp.max()) + 1
    rng = np.random.default_rng(11)
    I = rng.standard_normal((dev.N, 3)) + 1j * rng.standard_normal((dev.N, 3))
    L = rng.standard_normal((dev.N, 3)) + 1j * rng.standard_normal((dev.N, 3))
    g = dev.gradient_impedance(I, L, tp, P, reactive=reactive)
    ref = oc.gradient_impedance(I, L, tp, P, reactive=reactive)
    assert np.max(np.abs(g - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_forward_adjoint_gradient_chain(plate):
    m, rwg, dev, oc = plate
    k = 2 * math.pi / 0.1
    tp = _quadrants(m)
    theta = np.array([80.0, 120.0, 60.0, 150.0])
    dev.assemble(k, precision="fp64")
    dev.apply_impedance(theta[tp].astype(complex))
    v = oc.plane_wave_rhs([0, 0, -k], 1.0, [1, 0, 0])
    I, st = dev.gmres(v, tol=1e-12, maxiter=300)
    rng = np.random.default_rng(5)
    A = rng.standard_normal((5, dev.N)) + 1j * rng.standard_normal((5, dev.N))
    Q = A.conj().T @ A
    lam = solve_adjoint_rhs(dev, Q @ I, gmres_tol=1e-12, gmres_maxiter=300)
    Mp = precompute_patch_mass(m, rwg, PatchPartition(tp + 1, 4), device=dev)
    g = gradient_impedance(Mp, I, lam)
    # oracle: dense system, dense solves
    Z = oc.apply_impedance(oc.assemble_z(k), theta[tp].astype(complex))
    Io = np.linalg.solve(Z, v)
    lo = np.linalg.solve(Z.conj().T, Q @ Io)
    ref = oc.gradient_impedance(Io, lo, tp, 4)
    assert np.max(np.abs(g - ref)) <= 1e-8 * np.max(np.abs(ref))


def test_bad_partition_is_rejected(plate):
    m, rwg, dev, oc = plate
    tp = np.zeros(m.ntriangles, int)
    tp[3] = 7
    with pytest.raises(Exception):
        dev.gradient_impedance(np.ones(dev.N, complex), np.ones(dev.N, complex), tp, 4)
    with pytest.raises(ValueError):
        PatchPartition(np.zeros(m.ntriangles, int), 1)  # 1-based ids
