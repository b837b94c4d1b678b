"""Dipole and loop right-hand sides on the device against the oracle's
assemble_dipole / assemble_loop (Excitation.jl:2924-2977)."""
import math

import numpy as np
import pytest

import oracle as orc
from diffmom_b200 import (EFIEDevice, assemble_dipole, assemble_loop, assemble_multiple_excitations, build_rwg,
                          make_dipole, make_loop, make_plane_wave, make_rect_plate)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def plate():
    m = make_rect_plate(0.1, 0.1, 6, 6)
    rwg = build_rwg(m)
    dev = EFIEDevice(m, rwg)
    yield m, rwg, dev, orc.OracleCache(m, rwg, 3)
    dev.close()


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("kind", ["electric", "magnetic"])
def test_dipole_rhs_matches_oracle(plate, kind):
    m, rwg, dev, oc = plate
    d = make_dipole([0.03, -0.02, 0.12], [0, 0.3e-9j, 1.5e-9 + 0.4e-9j], [0, 0, 1], kind, 3e9)
    v = assemble_dipole(m, rwg, d, device=dev)
    ref = oc.dipole_rhs(d.position, d.moment, kind, d.frequency)
    assert _rel(v, ref) < 1e-12


def test_loop_rhs_matches_oracle_and_equivalent_dipole(plate):
    m, rwg, dev, oc = plate
    lp = make_loop([-0.04, 0.01, 0.14], [0, 1, 0], 0.012, 1.0 + 0.35j, 3e9)
    v = assemble_loop(m, rwg, lp, device=dev)
    ref = oc.dipole_rhs(lp.center, lp.equivalent_moment(), "magnetic", lp.frequency)
    assert _rel(v, ref) < 1e-12
    d = make_dipole(lp.center, lp.equivalent_moment(), lp.normal, "magnetic", lp.frequency)
    np.testing.assert_array_equal(v, assemble_dipole(m, rwg, d, device=dev))


def test_many_sources_one_launch(plate):
    m, rwg, dev, oc = plate
    rng = np.random.default_rng(5)
    R = 37
    pos = np.column_stack([rng.uniform(-0.1, 0.1, R), rng.uniform(-0.1, 0.1, R), rng.uniform(0.02, 0.3, R)])
    mom = rng.standard_normal((R, 3)) + 1j * rng.standard_normal((R, 3))
    types = ["magnetic" if i % 3 == 0 else "electric" for i in range(R)]
    freqs = rng.uniform(0.5e9, 4e9, R)
    V = dev.dipole_rhs(pos, mom, types, freqs)
    for r in range(R):
        ref = oc.dipole_rhs(pos[r], mom[r], types[r], freqs[r])
        assert _rel(V[:, r], ref) < 1e-12


def test_mixed_excitation_list(plate):
    m, rwg, dev, oc = plate
    k = 2 * math.pi * 3e9 / 299792458.0
    pw = make_plane_wave([0, 0, -k], 1.0, [1, 0, 0])
    d = make_dipole([0, 0, 0.1], [1e-9, 0, 0], [1, 0, 0], "electric", 3e9)
    lp = make_loop([0, 0, 0.1], [0, 0, 1], 0.01, 1.0, 3e9)
    V = assemble_multiple_excitations(m, rwg, [d, pw, lp], device=dev)
    assert _rel(V[:, 0], oc.dipole_rhs(d.position, d.moment, "electric", 3e9)) < 1e-12
    assert _rel(V[:, 1], oc.plane_wave_rhs(pw.k_vec, pw.E0, pw.pol)) < 1e-12
    assert _rel(V[:, 2], oc.dipole_rhs(lp.center, lp.equivalent_moment(), "magnetic", 3e9)) < 1e-12


def test_invalid_dipole_arguments_raise(plate):
    m, rwg, dev, oc = plate
    with pytest.raises(ValueError):
        dev.dipole_rhs([[0, 0, 0.1]], [[1, 0, 0]], ["scalar"], [1e9])
    with pytest.raises(Exception):
        dev.dipole_rhs([[0, 0, 0.1]], [[1, 0, 0]], ["electric"], [-1.0])
