"""Pattern-feed right-hand sides on the device against the oracle's
assemble_pattern_feed (Excitation.jl:3044-3071)."""
import math

import numpy as np
import pytest

import oracle as orc
from diffmom_b200 import (EFIEDevice, assemble_multiple_excitations, assemble_pattern_feed, build_rwg,
                          make_analytic_dipole_pattern_feed, make_dipole, make_pattern_feed, make_plane_wave,
                          make_rect_plate)

pytestmark = pytest.mark.gpu
FREQ = 3e9


@pytest.fixture(scope="module")
def plate():
    m = make_rect_plate(0.1, 0.1, 6, 6)
    rwg = build_rwg(m)
    dev = EFIEDevice(m, rwg)
    yield m, rwg, dev, orc.OracleCache(m, rwg, 3)
    dev.close()


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _oracle(oc, p):
    return oc.pattern_rhs(p.theta, p.phi, p.Ftheta, p.Fphi, p.frequency, p.phase_center,
                          p.convention == "exp_minus_iwt")


@pytest.mark.parametrize("kind", ["electric", "magnetic"])
def test_analytic_dipole_pattern_rhs(plate, kind):
    m, rwg, dev, oc = plate
    d = make_dipole([0.02, -0.01, 0.15], [0.2, 1j, 1.0], [0, 0, 1], kind, FREQ)
    pat = make_analytic_dipole_pattern_feed(d, np.linspace(0, 180, 19), np.arange(0, 360, 10),
                                            angles_in_degrees=True)
    v = assemble_pattern_feed(m, rwg, pat, device=dev)
    assert _rel(v, _oracle(oc, pat)) < 1e-12


@pytest.mark.parametrize("conv", ["exp_plus_iwt", "exp_minus_iwt"])
def test_random_pattern_nonuniform_grid(plate, conv):
    m, rwg, dev, oc = plate
    rng = np.random.default_rng(7)
    th = np.sort(rng.uniform(0.3, 2.8, 9))
    ph = np.sort(rng.uniform(0.1, 6.0, 11))  # the sources' directions cross the periodic seam
    F1 = rng.standard_normal((9, 11)) + 1j * rng.standard_normal((9, 11))
    F2 = rng.standard_normal((9, 11)) + 1j * rng.standard_normal((9, 11))
    pat = make_pattern_feed(th, ph, F1, F2, FREQ, phase_center=(0.01, 0.02, -0.12), convention=conv)
    v = dev.pattern_feed_rhs(pat)
    assert _rel(v, _oracle(oc, pat)) < 1e-12


def test_pattern_in_mixed_excitation_list(plate):
    m, rwg, dev, oc = plate
    k = 2 * math.pi * FREQ / 299792458.0
    d = make_dipole([0, 0, 0.1], [1e-9, 0, 0], [1, 0, 0], "electric", FREQ)
    pat = make_analytic_dipole_pattern_feed(d, np.linspace(0, math.pi, 7), np.linspace(0, 2 * math.pi, 8,
                                                                                     endpoint=False))
    pw = make_plane_wave([0, 0, -k], 1.0, [0, 1, 0])
    V = assemble_multiple_excitations(m, rwg, [pat, pw, d], device=dev)
    assert _rel(V[:, 0], _oracle(oc, pat)) < 1e-12
    assert _rel(V[:, 1], oc.plane_wave_rhs(pw.k_vec, pw.E0, pw.pol)) < 1e-12
    assert _rel(V[:, 2], oc.dipole_rhs(d.position, d.moment, "electric", FREQ)) < 1e-12
