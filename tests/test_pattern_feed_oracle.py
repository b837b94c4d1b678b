"""Pattern-feed sources on the CPU: the oracle's field (a restatement of
Excitation.jl:1170-1340, 1417-1460) against closed forms -- exact bilinear
data, the periodic phi seam, theta clamping -- and against the dipole field
it samples (make_analytic_dipole_pattern_feed, Excitation.jl:1468-1509;
the reference checks the same pairing, runtests.jl:4316-4324), plus the
constructor validation of make_pattern_feed."""
import math

import numpy as np
import pytest

import oracle as orc
from diffmom_b200 import make_analytic_dipole_pattern_feed, make_dipole, make_pattern_feed

FREQ = 3e9
K = 2 * math.pi * FREQ / 299792458.0


def _direct(points, Ft_fun, Fp_fun, pc=np.zeros(3)):
    d = np.atleast_2d(points) - pc
    R = np.linalg.norm(d, axis=1)
    th = np.arccos(np.clip(d[:, 2] / R, -1, 1))
    ph = np.arctan2(d[:, 1], d[:, 0]) % (2 * math.pi)
    et = np.stack([np.cos(th) * np.cos(ph), np.cos(th) * np.sin(ph), -np.sin(th)], 1)
    ep = np.stack([-np.sin(ph), np.cos(ph), 0 * ph], 1)
    return (Ft_fun(th, ph)[:, None] * et + Fp_fun(th, ph)[:, None] * ep) * (np.exp(-1j * K * R) / R)[:, None]


def test_bilinear_data_is_reproduced_exactly():
    th = np.linspace(0.1, 3.0, 13)
    ph = np.linspace(0.2, 5.9, 17)
    ft = lambda t, p: (1 + 2j) + (0.5 - 1j) * t + 0.25j * p + 0.1 * t * p
    fp = lambda t, p: (-0.3 + 0.7j) * t * p + 2.0
    T, P = np.meshgrid(th, ph, indexing="ij")
    rng = np.random.default_rng(4)
    dirs = []
    while len(dirs) < 40:
        t, p = rng.uniform(0.1, 3.0), rng.uniform(0.2, 5.9)
        dirs.append([math.sin(t) * math.cos(p), math.sin(t) * math.sin(p), math.cos(t)])
    pts = np.array(dirs) * rng.uniform(0.5, 3.0, (40, 1))
    E = orc.pattern_field(pts, th, ph, ft(T, P), fp(T, P), FREQ)
    ref = _direct(pts, ft, fp)
    assert np.max(np.abs(E - ref)) / np.max(np.abs(ref)) < 1e-13


def test_periodic_seam_and_theta_clamp():
    th = np.array([0.5, 1.0, 2.0])
    ph = np.array([0.5, 2.0, 4.0, 5.5])  # seam: 5.5 -> 0.5 + 2 pi
    Fa = np.zeros((3, 4), complex)
    Fa[:, 3] = 1.0                         # 1 at phi = 5.5, 0 at phi = 0.5 (+ 2 pi)
    Fb = np.ones((3, 4), complex) * (0.5 - 0.25j)
    span = 0.5 + 2 * math.pi - 5.5
    for p in (5.9, 6.2, 0.1, 0.3):
        for t in (0.2, 0.7, 2.6):           # below the grid, inside, above it
            r = np.array([[math.sin(t) * math.cos(p), math.sin(t) * math.sin(p), math.cos(t)]]) * 2.0
            E = orc.pattern_field(r, th, ph, Fa, Fb, FREQ)
            w = (p - 5.5) % (2 * math.pi)
            ref = _direct(r, lambda tt, pp: np.full_like(tt, 1 - w / span, dtype=complex),
                          lambda tt, pp: np.full_like(tt, 0.5 - 0.25j, dtype=complex))
            assert np.max(np.abs(E - ref)) < 1e-13 * np.max(np.abs(ref))


@pytest.mark.parametrize("kind", ["electric", "magnetic"])
def test_analytic_dipole_pattern_matches_dipole_far_field(kind):
    d = make_dipole([0.01, -0.02, 0.03], [0.3 + 0.1j, -0.2j, 1.0] if kind == "electric" else [0, 0.5, 1j],
                    [0, 0, 1], kind, FREQ)
    th = np.linspace(0, math.pi, 181)
    ph = np.arange(360) * math.pi / 180
    pat = make_analytic_dipole_pattern_feed(d, th, ph)
    rng = np.random.default_rng(9)
    u = rng.standard_normal((25, 3))
    pts = d.position + 100.0 * u / np.linalg.norm(u, axis=1, keepdims=True)  # 1000 wavelengths out
    E = orc.pattern_field(pts, pat.theta, pat.phi, pat.Ftheta, pat.Fphi, FREQ, pat.phase_center)
    Ed = orc.dipole_field(pts, d.position, d.moment, kind, FREQ)
    err = np.linalg.norm(E - Ed, axis=1) / np.linalg.norm(Ed, axis=1)
    assert err.max() < 2e-3


def test_exp_minus_iwt_conjugates_the_coefficients():
    th = np.linspace(0.1, 3.0, 5)
    ph = np.linspace(0.0, 5.0, 6)
    rng = np.random.default_rng(2)
    F = rng.standard_normal((5, 6)) + 1j * rng.standard_normal((5, 6))
    pts = rng.standard_normal((6, 3))
    a = orc.pattern_field(pts, th, ph, F, F, FREQ, conj_convention=True)
    b = orc.pattern_field(pts, th, ph, F.conj(), F.conj(), FREQ)
    np.testing.assert_array_equal(a, b)


def test_constructor_validation():
    F = np.ones((3, 3))
    with pytest.raises(ValueError):
        make_pattern_feed([0.0, 1.0], [0.0, 1.0, 2.0], F, F, FREQ)           # shape
    with pytest.raises(ValueError):
        make_pattern_feed([0.0, 2.0, 1.0], [0.0, 1.0, 2.0], F, F, FREQ)      # theta order
    with pytest.raises(ValueError):
        make_pattern_feed([0.0, 1.0, 4.0], [0.0, 1.0, 2.0], F, F, FREQ)      # theta > pi
    with pytest.raises(ValueError):
        make_pattern_feed([0.0, 1.0, 2.0], [0.0, 3.0, 2 * math.pi], F, F, FREQ)  # duplicate endpoint
    with pytest.raises(ValueError):
        make_pattern_feed([0.0, 1.0, 2.0], [0.0, 1.0, 2.0], F, F, -1.0)
    with pytest.raises(ValueError):
        make_pattern_feed([0.0, 1.0, 2.0], [0.0, 1.0, 2.0], F, F, FREQ, convention="exp_iwt")
    p = make_pattern_feed([0, 90, 180], [0, 120, 240], F, F, FREQ, angles_in_degrees=True,
                          convention=":exp_minus_iwt")
    assert p.convention == "exp_minus_iwt" and abs(p.theta[-1] - math.pi) < 1e-15
