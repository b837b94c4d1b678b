"""Uneven batch of impedance-loaded surfaces (many lanes, largest first)
against one-surface-at-a-time solves, and the far-pair tile autotuner's
shapes against each other."""
import math

import numpy as np
import pytest

from diffmom_b200 import (EFIEDevice, SphGrid, bistatic_rcs, build_rwg, compute_farfield, make_rect_plate,
                          solve_surfaces)
from diffmom_b200.workloads import impedance_surface_batch

pytestmark = pytest.mark.gpu
C0 = 299792458.0
K3 = 2 * math.pi * 3e9 / C0


def test_far_tile_shapes_identical():
    """Every RWG tile width of the far-pair kernel writes the same Z bit for
    bit, and Z is bitwise symmetric (the four triangle pairs of an entry are
    summed in an order that does not depend on which index is the row)."""
    m = make_rect_plate(0.1, 0.1, 14, 9)
    dev = EFIEDevice(m, build_rwg(m))
    for prec, widths in (("fp64", (16, 32, 0)), ("mixed", (32, 64, 0))):
        ref = None
        for w in widths:
            dev.set_option("far_tile", w)
            Z = dev.assemble(K3, precision=prec, copy_out=True)
            assert dev.far_tile() in widths[:2]
            assert np.array_equal(Z, Z.T), (prec, w)
            if ref is None:
                ref = Z
            else:
                assert np.array_equal(Z, ref), (prec, w)
    with pytest.raises(Exception):
        dev.set_option("far_tile", 8)
    dev.set_option("far_tile", 64)
    with pytest.raises(Exception):
        dev.assemble(K3, precision="fp64")  # 64 is an FP32 width only
    dev.set_option("far_tile", 0)
    dev.close()


def test_surface_batch_matches_single_solves():
    surf = impedance_surface_batch(count=6, seed=5, n_range=(150, 1200))
    res = solve_surfaces(surf, 3e9, lanes=3, precision="fp64", gmres_tol=1e-10, return_currents=True)
    assert res.device_ms > 0 and np.all(res.latency_ms > 0) and np.all(res.true_residual <= 1e-9)
    # one batch-wide assembly (far tiles of every surface in one launch)
    assert 0 < res.assembly_ms < res.device_ms
    for i, sf in enumerate(surf):
        dev = EFIEDevice(sf.mesh, sf.rwg)
        dev.assemble(K3)
        dev.apply_impedance(sf.zs)
        e = sf.excitation
        v = dev.plane_wave_rhs([e.k_vec], [e.E0], [e.pol])[:, 0]
        P = dev.build_nearfield(math.inf, "lu")
        x, st = dev.gmres(v, tol=1e-10, maxiter=300, preconditioner=P)
        x = np.asarray(x).reshape(-1)
        rh = -np.asarray(e.k_vec) / np.linalg.norm(e.k_vec)
        E = compute_farfield(dev, SphGrid(rh[None], np.zeros(1), np.zeros(1), np.ones(1)), x)
        sig = bistatic_rcs(np.asarray(E).reshape(3, -1))[0]
        # the batched assembly writes the same Z as the surface's own assembly
        assert np.linalg.norm(res.currents[i] - x) <= 1e-8 * np.linalg.norm(x)
        assert abs(res.sigma[i] - sig) <= 1e-8 * sig
        dev.close()
    one = solve_surfaces(surf, 3e9, lanes=1, precision="fp64", gmres_tol=1e-10)
    assert np.allclose(one.sigma, res.sigma, rtol=1e-12, atol=0)
    mixed = solve_surfaces(surf, 3e9, lanes=3, precision="mixed", gmres_tol=1e-6)
    rel = np.abs(mixed.sigma - res.sigma) / res.sigma
    print(f"N {res.N}; mixed vs FP64 RCS error max {rel.max():.2e}; lanes=3 {res.device_ms:.1f} ms, "
          f"lanes=1 {one.device_ms:.1f} ms (FP64)")
    assert np.all(mixed.true_residual <= 1e-6)
    assert rel.max() <= 1e-3
