"""Parity at the benchmarked sizes (GPU), through the C ABI, against the CPU
oracle (oracle/efie_oracle.c: the C restatement of the reference's FP64
algorithm) at full size:

* the 7,680-RWG sphere (r = 0.5 lambda at 3 GHz, icosphere level 4, one
  x-polarised wave along -z): FP64 Z entrywise (EFIE.jl:699-753), FP64
  currents and the 181-point phi = 0 bistatic RCS (FarField.jl:425-611,
  Diagnostics.jl:460-474) to 1e-8, the mixed path (FP32 far pairs, complex64 Z,
  GMRES to 1e-6 on the FP64 residual) to 1e-4 in RCS, and the Mie series as the
  physics gate (runtests.jl:5176-5240);
* the 10,680-RWG plate (0.3 m, 60 x 60 cells, 3 GHz) with 32 seeded incidences
  of the headline sweep: per incidence, the mixed batched currents and
  monostatic sigma within 1e-4 of the oracle's LAPACK solve, the FP64 path's
  currents within 1e-8.
"""
import math

import numpy as np
import pytest
import scipy.linalg as sla

import oracle as orc
from diffmom_b200 import (EFIEDevice, bistatic_rcs, build_rwg, make_icosphere, make_plane_wave,
                          make_rect_plate, monostatic_rcs_sweep, phi_cut_grid)

pytestmark = pytest.mark.gpu

C0 = 299792458.0
F = 3e9
LAM = C0 / F
K = 2 * math.pi / LAM


def _threads():
    import os
    return min(os.cpu_count() or 1, orc.max_threads())


@pytest.fixture(scope="module")
def sphere_c2():
    m = make_icosphere(0.5 * LAM, 4)
    r = build_rwg(m)
    assert r.nedges == 7680
    c = orc.OracleCache(m, r, 3)
    Zo = c.assemble_z(K, nthreads=_threads())
    vo = c.plane_wave_rhs([0.0, 0.0, -K], 1.0, [1.0, 0.0, 0.0])
    Io = sla.solve(Zo, vo, check_finite=False)
    grid = phi_cut_grid(0.0, np.arange(0, 181, 1.0))
    G = c.radiation_vectors(grid.rhat, K)
    so = bistatic_rcs((G @ Io).reshape(-1, 3).T)
    return m, r, Zo, vo, Io, grid, so


def test_c2_sphere_fp64_against_oracle(sphere_c2):
    m, r, Zo, vo, Io, grid, so = sphere_c2
    dev = EFIEDevice(m, r)
    Z = dev.assemble(K, precision="fp64", copy_out=True)
    zmax = np.max(np.abs(Zo))
    big = np.abs(Zo) > 1e-4 * zmax
    rel = np.max(np.abs(Z[big] - Zo[big]) / np.abs(Zo[big]))
    small = np.max(np.abs(Z[~big] - Zo[~big])) if (~big).any() else 0.0
    print(f"C2 FP64 Z: entrywise rel {rel:.2e}, small entries abs {small / zmax:.2e} of max|Z|")
    assert rel < 1e-10 and small < 1e-14 * zmax
    del Z
    # currents and RCS: the FP64 direct solve (LDL^T of Z + FP64 refinement)
    v = dev.plane_wave_rhs([[0.0, 0.0, -K]], [1.0], [[1.0, 0.0, 0.0]])[:, 0]
    assert np.linalg.norm(v - vo) <= 1e-13 * np.linalg.norm(vo)
    I, berr = dev.solve_direct(v)
    I = I.reshape(-1)
    cerr = np.linalg.norm(I - Io) / np.linalg.norm(Io)
    sg = bistatic_rcs(dev.farfield(grid.rhat, I, k=K))
    serr = np.max(np.abs(sg - so) / so)
    # and FP64 GMRES with the reference's 1-lambda near-field preconditioner
    P = dev.build_nearfield(1.0 * LAM, "lu")
    Ig, st = dev.gmres(v, tol=1e-11, maxiter=300, preconditioner=P, precond_side="left")
    Ig = Ig.reshape(-1)
    gerr = np.linalg.norm(Ig - Io) / np.linalg.norm(Io)
    print(f"C2 FP64: direct currents {cerr:.2e}, RCS {serr:.2e} (181 directions); NF-GMRES "
          f"{st.niter} iterations, currents {gerr:.2e}, true residual {st.true_residual:.2e}")
    assert cerr < 1e-8 and serr < 1e-8
    assert st.solved and st.true_residual <= 1e-11 and gerr < 1e-8
    # physics gate: Mie series at this size (runtests.jl:5237-5240 thresholds)
    a = float(np.mean(np.linalg.norm(m.xyz - m.xyz.mean(axis=0), axis=1)))
    mie = np.array([orc.mie_bistatic_rcs_pec(K, a, [0, 0, -1], [1, 0, 0], d) for d in grid.rhat])
    dB = 10 * np.log10(sg) - 10 * np.log10(mie)
    print(f"C2 vs Mie: MAE {np.mean(np.abs(dB)):.3f} dB, max {np.max(np.abs(dB)):.3f} dB")
    assert np.mean(np.abs(dB)) < 0.5 and np.max(np.abs(dB)) < 1.2
    dev.close()


def test_c2_sphere_mixed_against_oracle(sphere_c2):
    m, r, Zo, vo, Io, grid, so = sphere_c2
    dev = EFIEDevice(m, r)
    Zm = dev.assemble(K, precision="mixed", copy_out=True)
    zerr = np.linalg.norm(Zm - Zo) / np.linalg.norm(Zo)
    del Zm
    res = dev.solve_many(K, [[0.0, 0.0, -K]], [[1.0, 0.0, 0.0]], precision="mixed", preconditioner="lu",
                         cutoff=1.0 * LAM, tol=1e-6, maxiter=300, precond_side="right")
    st = res[1]
    I = dev.currents()[:, 0]
    sg = bistatic_rcs(dev.farfield(grid.rhat, I, k=K))
    cerr = np.linalg.norm(I - Io) / np.linalg.norm(Io)
    serr = np.max(np.abs(sg - so) / so)
    print(f"C2 mixed: Z normwise {zerr:.2e}, currents {cerr:.2e}, RCS {serr:.2e} (181 directions), "
          f"true residual {st.true_residual:.2e}")
    assert zerr < 2e-6
    assert st.solved and st.true_residual <= 1e-6
    assert serr < 1e-4 and cerr < 1e-4
    dev.close()


def _waves(R, seed):
    rng = np.random.default_rng(seed)
    th = np.deg2rad(rng.uniform(0.0, 80.0, R))
    ph = np.deg2rad(rng.uniform(0.0, 360.0, R))
    rhat = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], 1)
    tha = np.stack([np.cos(th) * np.cos(ph), np.cos(th) * np.sin(ph), -np.sin(th)], 1)
    pha = np.stack([-np.sin(ph), np.cos(ph), np.zeros(R)], 1)
    pol = np.where((np.arange(R) % 2 == 0)[:, None], tha, pha)
    return -K * rhat, pol


def test_c3_plate_sweep_against_oracle():
    # 32 incidences of the headline workload (seed 20260001: the first 32 of
    # the bench's draw use another seed, the statistics are the same)
    m = make_rect_plate(0.3, 0.3, 60, 60)
    r = build_rwg(m)
    assert r.nedges == 10680
    R = 32
    kv, pol = _waves(R, 20260032)
    c = orc.OracleCache(m, r, 3)
    Zo = c.assemble_z(K, nthreads=_threads())
    V = np.stack([c.plane_wave_rhs(kv[i], 1.0, pol[i]) for i in range(R)], 1)
    Io = sla.lu_solve(sla.lu_factor(Zo, overwrite_a=True, check_finite=False), V, check_finite=False)
    del Zo
    so = np.empty(R)
    for i in range(R):
        E = c.radiation_vectors(-kv[i] / K, K) @ Io[:, i]
        so[i] = 4 * math.pi * np.sum(np.abs(E) ** 2)
    exc = [make_plane_wave(kv[i], 1.0, pol[i]) for i in range(R)]
    dev = EFIEDevice(m, r)
    rm = monostatic_rcs_sweep(m, F, exc, precision="mixed", gmres_tol=1e-6, device=dev, rwg=r,
                              return_currents=True)
    cur = np.linalg.norm(rm.currents - Io, axis=0) / np.linalg.norm(Io, axis=0)
    sg = np.abs(rm.sigma - so) / so
    print(f"C3 mixed batched, {R} incidences: {rm.gmres_iters} iterations, true residual "
          f"{rm.true_residual:.2e}; per incidence currents max {cur.max():.2e}, sigma max {sg.max():.2e}")
    assert rm.true_residual <= 1e-6
    assert cur.max() <= 1e-4 and sg.max() <= 1e-4
    r64 = monostatic_rcs_sweep(m, F, exc, precision="fp64", gmres_tol=1e-11, device=dev, rwg=r,
                               return_currents=True)
    cur64 = np.linalg.norm(r64.currents - Io, axis=0) / np.linalg.norm(Io, axis=0)
    sg64 = np.abs(r64.sigma - so) / so
    print(f"C3 FP64: {r64.gmres_iters} iterations, true residual {r64.true_residual:.2e}; currents max "
          f"{cur64.max():.2e}, sigma max {sg64.max():.2e}")
    assert r64.true_residual <= 1e-11
    assert cur64.max() <= 1e-8 and sg64.max() <= 1e-8
    dev.close()
