"""GPU path against the committed golden fixtures (written by the oracle,
tests/golden/make_golden.py): the C1 plate's Z, currents, bistatic RCS cut
and monostatic sweep, and sampled entries of the C2 sphere's Z."""
import math
from pathlib import Path

import numpy as np
import pytest

from diffmom_b200 import (EFIEDevice, SphGrid, bistatic_rcs, build_rwg, compute_farfield, make_icosphere,
                          make_plane_wave, make_rect_plate, monostatic_rcs_sweep)

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).parent / "golden"
C0 = 299792458.0


def _entrywise(a, ref, rel=1e-10):
    # relative error for entries above 1e-4 max|ref|, absolute 1e-14 max|ref| below
    big = np.abs(ref) >= 1e-4 * np.abs(ref).max()
    assert np.max(np.abs(a[big] - ref[big]) / np.abs(ref[big])) < rel
    assert np.max(np.abs(a[~big] - ref[~big]), initial=0.0) < 1e-14 * np.abs(ref).max()


def test_c1_plate_against_fixture():
    g = np.load(GOLD / "c1_plate.npz")
    k = float(g["k"])
    m = make_rect_plate(0.1, 0.1, 6, 6)
    rwg = build_rwg(m)
    dev = EFIEDevice(m, rwg)
    Z = dev.assemble(k, copy_out=True)
    _entrywise(Z, g["Z"])
    v = dev.plane_wave_rhs([[0, 0, -k]], [1.0], [[1, 0, 0]])[:, 0]
    assert np.linalg.norm(v - g["v"]) <= 1e-13 * np.linalg.norm(g["v"])
    I, _ = dev.solve_direct(v)
    I = np.asarray(I).reshape(-1)
    assert np.linalg.norm(I - g["I"]) <= 1e-8 * np.linalg.norm(g["I"])
    th = g["theta"]
    grid = SphGrid(np.stack([np.sin(th), np.zeros_like(th), np.cos(th)], 1), th, np.zeros_like(th),
                   np.ones_like(th))
    E = compute_farfield(dev, grid, I, k=k)
    sig = bistatic_rcs(np.asarray(E).reshape(3, -1))
    assert np.max(np.abs(sig - g["sigma_cut"]) / g["sigma_cut"]) < 1e-8
    exc = [make_plane_wave(g["kvecs"][i], 1.0, g["pols"][i]) for i in range(6)]
    res = monostatic_rcs_sweep(m, k * C0 / (2 * math.pi), exc, precision="fp64", gmres_tol=1e-12, device=dev,
                               rwg=rwg, return_currents=True)
    assert np.max(np.abs(res.sigma - g["sigma_mono"]) / g["sigma_mono"]) < 1e-8
    assert np.linalg.norm(res.currents - g["I_mono"]) <= 1e-8 * np.linalg.norm(g["I_mono"])
    dev.close()


def test_c2_sphere_entries_against_fixture():
    g = np.load(GOLD / "c2_sphere_sample.npz")
    lam = C0 / 3e9
    m = make_icosphere(0.5 * lam, 4)
    dev = EFIEDevice(m, build_rwg(m))
    k = float(g["k"])
    dev.assemble(k)
    z = dev.entries(g["m"], g["n"])
    _entrywise(z, g["z"])
    v = dev.plane_wave_rhs([[0, 0, -k]], [1.0], [[1, 0, 0]])[:, 0]
    assert np.linalg.norm(v - g["v"]) <= 1e-13 * np.linalg.norm(g["v"])
    dev.close()
