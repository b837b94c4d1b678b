"""Dipole and loop sources on the CPU: the oracle's field against the
reference's analytic checks (runtests.jl:7001-7040) and a 60-digit closed
form, plus the constructor validation of make_dipole / make_loop
(runtests.jl:5666-5679)."""
import math

import numpy as np
import pytest

import oracle as orc
from diffmom_b200 import make_dipole, make_loop

FREQ = 1.0e9
K = 2 * math.pi * FREQ / 299792458.0
ETA0 = 376.730313668
EPS0 = 8.854187817e-12


def test_magnetic_dipole_far_field():
    m = np.array([0, 0, 1e-4], dtype=complex)
    E = orc.dipole_field(np.array([[5.0, 0, 0]]), np.zeros(3), m, "magnetic", FREQ)[0]
    ref = ETA0 * K ** 2 * m[2] * np.exp(-1j * K * 5.0) / (4 * math.pi * 5.0)
    assert abs(E[1] - ref) / abs(ref) < 0.03


def test_electric_dipole_broadside_and_quasistatic():
    p = np.array([0, 0, 1e-12], dtype=complex)
    E = orc.dipole_field(np.array([[8.0, 0, 0]]), np.zeros(3), p, "electric", FREQ)[0]
    ref = p[2] * K ** 2 * np.exp(-1j * K * 8.0) / (4 * math.pi * EPS0 * 8.0)
    assert abs(E[2] - ref) / abs(ref) < 0.03
    Eq = orc.dipole_field(np.array([[0, 0, 0.5]]), np.zeros(3), p, "electric", 1.0e6)[0]
    st = 2 * p[2] / (4 * math.pi * EPS0 * 0.5 ** 3)
    assert abs(Eq[2].real - st.real) / abs(st.real) < 0.05


def test_loop_is_equivalent_magnetic_dipole():
    loop = make_loop([0, 0, 0], [0, 0, 1], 0.01, 2.0, FREQ)
    m = np.array([0, 0, 2.0 * math.pi * 0.01 ** 2], dtype=complex)
    np.testing.assert_array_equal(loop.equivalent_moment(), m)
    E1 = orc.dipole_field(np.array([[5.0, 0, 0]]), loop.center, loop.equivalent_moment(), "magnetic", FREQ)
    E2 = orc.dipole_field(np.array([[5.0, 0, 0]]), np.zeros(3), m, "magnetic", FREQ)
    np.testing.assert_array_equal(E1, E2)


def _closed_form(mp, r, pos, mom, magnetic, freq):
    mp.mp.dps = 60
    eps0 = mp.mpf("8.854187817e-12")
    mu0 = 4 * mp.pi * mp.mpf("1e-7")
    eta0, c0 = mp.sqrt(mu0 / eps0), 1 / mp.sqrt(eps0 * mu0)
    k = 2 * mp.pi * mp.mpf(freq) / c0
    d = [mp.mpf(r[i]) - mp.mpf(pos[i]) for i in range(3)]
    p = [mp.mpc(complex(x)) for x in mom]
    R = mp.sqrt(sum(x * x for x in d))
    cross = lambda a, b: [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]
    ph = mp.exp(-1j * k * R)
    if not magnetic:
        t1 = cross(cross(d, p), d)
        dp = sum(d[i] * p[i] for i in range(3))
        return [((k * k * t1[i] / R ** 2) + (3 * d[i] * dp / R ** 2 - p[i]) * (1 / R ** 2 + 1j * k / R)) * ph
                / (4 * mp.pi * eps0 * R) for i in range(3)]
    a = cross(p, d)
    f = eta0 / (4 * mp.pi) * (k * k / R - 1j * k / R ** 2) * ph
    return [f * a[i] / R for i in range(3)]


@pytest.mark.parametrize("magnetic", [False, True])
def test_dipole_field_against_extended_precision(magnetic):
    mp = pytest.importorskip("mpmath")
    rng = np.random.default_rng(11 + magnetic)
    pos = np.array([0.03, -0.02, 0.12])
    mom = (rng.standard_normal(3) + 1j * rng.standard_normal(3)) * (1e-4 if magnetic else 1e-9)
    pts = rng.uniform(-0.3, 0.3, (12, 3))
    E = orc.dipole_field(pts, pos, mom, "magnetic" if magnetic else "electric", 3e9)
    worst = 0.0
    for i in range(pts.shape[0]):
        ref = np.array([complex(z) for z in _closed_form(mp, pts[i], pos, mom, magnetic, 3e9)])
        worst = max(worst, np.linalg.norm(E[i] - ref) / np.linalg.norm(ref))
    assert worst < 1e-13


def test_dipole_field_at_source_is_zero():
    E = orc.dipole_field(np.array([[0.1, 0.2, 0.3]]), np.array([0.1, 0.2, 0.3]), np.ones(3, complex), "electric")
    assert np.all(E == 0)


def test_constructor_validation():
    with pytest.raises(ValueError):
        make_dipole([0, 0, 0], [1, 0, 0], [1, 0, 0], "electric", math.inf)
    with pytest.raises(ValueError):
        make_loop([0, 0, 0], [0, 0, 1], -0.1, 1.0, FREQ)
    with pytest.raises(ValueError):
        make_dipole([0, 0, 0], [1, 0, 0], [1, 1, 0], "electric", FREQ)
    with pytest.raises(ValueError):
        make_dipole([0, 0, 0], [1, 0, 0], [1, 0, 0], "quadrupole", FREQ)
    with pytest.raises(ValueError):
        make_loop([0, 0, 0], [0, 0, 2], 0.1, 1.0, FREQ)
    with pytest.raises(ValueError):
        make_loop([0, 0, 0], [0, 0, 1], 0.1, complex(math.nan, 0), FREQ)
    d = make_dipole([0, 0, 0], [1, 0, 0], [1, 0, 0], ":magnetic")
    assert d.type == "magnetic" and d.frequency == 1e9
