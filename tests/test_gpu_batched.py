"""Many right-hand sides: the tensor-core complex GEMM Z X, the panel-blocked
near-field solves and block GMRES with FP64-residual refinement, each checked
against its FP64-accumulated counterpart on the same inputs."""
import math

import numpy as np
import pytest

from diffmom_b200 import EFIEDevice, build_rwg, make_rect_plate

pytestmark = pytest.mark.gpu

C0 = 299792458.0
K3 = 2 * math.pi * 3e9 / C0


def _plate(n, side=0.1):
    m = make_rect_plate(side, side, n, n)
    return EFIEDevice(m, build_rwg(m))


def _rand(N, R, seed):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.standard_normal((N, R)) + 1j * rng.standard_normal((N, R)))


def _waves(k, R, seed):
    # theta in [0, 80) deg, phi in [0, 360) deg; half theta-, half phi-polarised
    rng = np.random.default_rng(seed)
    th = np.deg2rad(rng.uniform(0, 80, R))
    ph = np.deg2rad(rng.uniform(0, 360, R))
    rhat = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], 1)
    tha = np.stack([np.cos(th) * np.cos(ph), np.cos(th) * np.sin(ph), -np.sin(th)], 1)
    pha = np.stack([-np.sin(ph), np.cos(ph), np.zeros(R)], 1)
    pol = np.where((np.arange(R) % 2 == 0)[:, None], tha, pha)
    return -k * rhat, np.ones(R), pol


def test_tensor_core_zx_matches_fp64_accumulation():
    dev = _plate(24)  # 1,680 RWG: K = 6.6 panels of 256, ragged edges in M, K and R
    dev.assemble(K3, precision="mixed")
    dev.set_option("exact_krylov", 0)
    for R in (64, 300):
        X = _rand(dev.N, R, R)
        dev.set_option("tc_min_rhs", 1 << 30)
        Y64 = dev.matvec(X)
        dev.set_option("tc_min_rhs", 64)
        Ytc = dev.matvec(X)
        err = np.linalg.norm(Ytc - Y64, axis=0) / np.linalg.norm(Y64, axis=0)
        print(f"R={R}: tensor-core Z X max column error {err.max():.2e}")
        # 3xTF32 operands (~2^-22) with FP32 accumulation in TMEM over
        # K'' = 6 x 1,792 floats
        assert err.max() < 5e-5
    dev.close()


@pytest.mark.parametrize("scheme,tol", [(0, 1e-12), (1, 2e-11)])
def test_int8_product_with_split_tail_tiles(scheme, tol):
    # 4,720 RWG x 600 columns: 74 x 3 = 222 output tiles on 148 SMs -- one
    # data-parallel wave and a tail whose tiles are split between CTAs and
    # summed by the fixup kernel.  scheme 0: residues modulo 13 moduli (CRT);
    # 1: seven-bit slices
    dev = _plate(40, side=0.3)
    dev.assemble(K3, precision="mixed")
    dev.set_option("tc_min_rhs", 1 << 30)
    dev.set_option("int8_scheme", scheme)
    X = _rand(dev.N, 600, 9)
    X[:, 7] *= 1e-30  # column scaling
    Y = dev.matvec(X)
    dev.set_option("tensor_cores", 0)
    Ys = dev.matvec(X)
    dev.set_option("tensor_cores", 1)
    err = np.linalg.norm(Y - Ys, axis=0) / np.linalg.norm(Ys, axis=0)
    print(f"scheme {scheme}: split-tail int8 product vs SIMT FP64: max column error {err.max():.2e}")
    assert err.max() <= tol
    for j in (0, 7, 255, 256, 599):
        y = dev.matvec(np.ascontiguousarray(X[:, j]))
        assert np.linalg.norm(Y[:, j] - y) <= tol * np.linalg.norm(y)
    np.testing.assert_array_equal(Y, dev.matvec(X))  # deterministic
    dev.close()


def test_int8_tile_candidates_identical():
    """The residue-scheme int8 product on one-SM 64 x 256 complex tiles and on
    CTA-pair 128 x 256 tiles (a two-CTA cluster, tcgen05 cta_group::2) writes
    the same bits: whole tiles, a stream-K tail of pair tiles (600 columns),
    four column tiles per row (1,024) and a single ragged one (100)."""
    dev = _plate(40, side=0.3)  # 4,720 RWG: 37 pair rows of tiles, ragged last
    dev.assemble(K3, precision="mixed")
    dev.set_option("tc_min_rhs", 1 << 30)
    for R in (600, 1024, 100):
        X = _rand(dev.N, R, 11 + R)
        out = {}
        for pin in (1, 2, 0):
            dev.set_option("tune_int8_tile", pin)
            out[pin] = dev.matvec(X)
        assert np.array_equal(out[1], out[2]), R
        assert np.array_equal(out[1], out[0]), R
    dev.set_option("tune_int8_tile", 0)
    with pytest.raises(Exception):
        dev.set_option("tune_int8_tile", 3)
    dev.close()


def test_int8_residue_scheme_krylov_class():
    # the Krylov operator of the many-RHS solves uses 12 moduli (fewer bits
    # for X, ~1e-11 normwise): right-preconditioned block GMRES with either
    # scheme meets the FP64 criterion in the same number of iterations, and the
    # true residual formed from the stored products (13 moduli) matches an
    # explicit b - Z x
    dev = _plate(30)
    dev.assemble(K3, precision="mixed")
    P = dev.build_nearfield(0.15 * C0 / 3e9, "lu")
    B = _rand(dev.N, 64, 4)
    its = {}
    for scheme in (0, 1):
        dev.set_option("int8_scheme", scheme)
        X, st = dev.gmres(B, tol=1e-8, maxiter=200, preconditioner=P, precond_side="right")
        rel = np.linalg.norm(B - dev.matvec(np.asfortranarray(X)), axis=0) / np.linalg.norm(B, axis=0)
        print(f"scheme {scheme}: {st.niter} iterations, reported true residual {st.true_residual:.2e}, "
              f"explicit {rel.max():.2e}")
        assert st.solved and rel.max() <= 1e-8
        assert abs(rel.max() - st.true_residual) <= 1e-2 * st.true_residual + 1e-11
        its[scheme] = st.niter
    assert abs(its[0] - its[1]) <= 2
    dev.close()


def test_fp64_accumulated_zx_matches_column_products():
    # the FP64-accurate Z X of the refinement residuals (int8 tensor-core
    # slices for complex64 Z from 32 right-hand sides, else SIMT FP64) against
    # the one-column FP64 product; ragged M and R
    dev = _plate(24)
    dev.assemble(K3, precision="mixed")
    dev.set_option("tc_min_rhs", 1 << 30)
    for R in (70, 300):
        X = _rand(dev.N, R, 5)
        Y = dev.matvec(X)
        dev.set_option("tensor_cores", 0)
        Ys = dev.matvec(X)
        dev.set_option("tensor_cores", 1)
        worst = 0.0
        for j in (0, R // 2, R - 1):
            y = dev.matvec(np.ascontiguousarray(X[:, j]))
            worst = max(worst, np.linalg.norm(Y[:, j] - y) / np.linalg.norm(y))
            assert np.linalg.norm(Ys[:, j] - y) <= 1e-13 * np.linalg.norm(y)
        print(f"R={R}: int8-slice FP64 product vs one-column FP64 {worst:.2e}, "
              f"vs SIMT FP64 {np.max(np.linalg.norm(Y - Ys, axis=0) / np.linalg.norm(Ys, axis=0)):.2e}")
        assert worst <= 2e-11
    dev.close()


def test_one_column_blocked_sweeps_match_chained_sweeps():
    # 4,720 RWG: five 1024-row blocks, the last one ragged.  One column of a
    # complex64 factor runs the blocked sweeps (FP64-product block inverses),
    # two columns the flag-ordered 64-row chain: same solve to FP32 level
    dev = _plate(40, side=0.3)
    dev.assemble(K3, precision="mixed")
    dev.build_nearfield(float("inf"), "lu")
    X = _rand(dev.N, 2, 3)
    Y2 = dev.nf_apply(X)
    for j in (0, 1):
        y1 = dev.nf_apply(np.ascontiguousarray(X[:, j]))
        err = np.linalg.norm(y1 - Y2[:, j]) / np.linalg.norm(Y2[:, j])
        res = np.linalg.norm(dev.matvec(y1) - X[:, j]) / np.linalg.norm(X[:, j])
        print(f"column {j}: blocked vs chained {err:.2e}, residual with Z {res:.2e}")
        assert err < 1e-5 and res < 1e-3
    np.testing.assert_array_equal(dev.nf_apply(np.ascontiguousarray(X[:, 0])),
                                  dev.nf_apply(np.ascontiguousarray(X[:, 0])))  # deterministic
    dev.close()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batched_nearfield_solve_matches_column_solves(precision):
    dev = _plate(24)
    dev.assemble(K3, precision=precision)
    dev.build_nearfield(0.05, "lu")
    for R in (8, 37, 200):
        X = _rand(dev.N, R, 7 + R)
        Yb = dev.nf_apply(X)
        cols = sorted({0, R // 2, R - 1})
        Ys = np.stack([dev.nf_apply(X[:, j]) for j in cols], 1)
        err = np.linalg.norm(Yb[:, cols] - Ys) / np.linalg.norm(Ys)
        print(f"{precision} R={R}: batched vs column solves {err:.2e}")
        assert err < (2e-5 if precision == "mixed" else 1e-12)
    dev.close()


@pytest.mark.parametrize("exact", [0, 1])
@pytest.mark.parametrize("side", ["left", "right"])
def test_block_gmres_many_plane_waves(side, exact):
    # 1,680 RWG plate (1 lambda), 256 incidences, complex64 Z, full c64 LDL^T as
    # the preconditioner: the Krylov products run on the tensor cores, the
    # returned currents must meet 1e-6 on the FP64 residual and match the FP64
    # solution of the same systems
    dev = _plate(24)
    kv, e0, pol = _waves(K3, 256, 20260001)
    dev.assemble(K3, precision="fp64")
    V = dev.plane_wave_rhs(kv, e0, pol)
    dev.build_nearfield(float("inf"), "lu")
    x64, st64 = dev.gmres(V, tol=1e-10, maxiter=100, preconditioner=dev.preconditioner)
    dev.assemble(K3, precision="mixed")
    dev.set_option("exact_krylov", exact)
    P = dev.build_nearfield(float("inf"), "lu")
    x, st = dev.gmres(V, tol=1e-6, maxiter=100, preconditioner=P, precond_side=side)
    err = np.linalg.norm(x - x64, axis=0) / np.linalg.norm(x64, axis=0)
    print(f"{side}, exact Krylov product {exact}: {st.niter} iterations, {st.restarts} refinement cycles, "
          f"true residual "
          f"{st.true_residual:.2e}, max current error vs FP64 {err.max():.2e}")
    assert st.solved
    # the unpreconditioned FP64 residual is the criterion on either side: a left-
    # preconditioned system that stopped on its preconditioned residual is
    # refined until ||b - Z x|| / ||b|| <= 1e-6
    assert st.true_residual <= 1e-6
    assert err.max() < 1e-4
    # the reported true residual -- formed from the stored Krylov products when
    # they are the FP64-accurate ones -- against b - Z x from a separate
    # FP64-accurate product through the public matvec
    dev.set_option("exact_krylov", 1)  # the public product then has every slice level
    Zx = dev.matvec(np.asfortranarray(x))
    explicit = np.max(np.linalg.norm(V - Zx, axis=0) / np.linalg.norm(V, axis=0))
    # both come from products accurate to ~1e-12 of |Z||x|: they agree to that
    # absolute level, five orders below the 1e-6 tolerance
    assert abs(explicit - st.true_residual) <= 1e-2 * st.true_residual + 2e-11
    dev.close()


def test_monostatic_sweep_matches_oracle():
    # C1 plate (72 triangles, 96 RWG), six incidences: currents by dense
    # solves of the oracle's Z, far field by its radiation vectors
    import oracle as orc
    from diffmom_b200 import make_plane_wave, monostatic_rcs_sweep
    m = make_rect_plate(0.1, 0.1, 6, 6)
    rwg = build_rwg(m)
    k = 2 * math.pi / 0.1
    kv, e0, pol = _waves(k, 6, 3)
    exc = [make_plane_wave(kv[i], 1.0, pol[i]) for i in range(6)]
    res = monostatic_rcs_sweep(m, k * C0 / (2 * math.pi), exc, precision="fp64", gmres_tol=1e-12,
                               rwg=rwg, return_currents=True)
    oc = orc.OracleCache(m, rwg, 3)
    Z = oc.assemble_z(k)
    sig = []
    for i in range(6):
        I = np.linalg.solve(Z, oc.plane_wave_rhs(kv[i], 1.0, pol[i]))
        G = oc.radiation_vectors(-kv[i] / k, k)
        E = G @ I
        sig.append(4 * math.pi * np.sum(np.abs(E) ** 2))
        assert np.linalg.norm(res.currents[:, i] - I) <= 1e-8 * np.linalg.norm(I)
    sig = np.array(sig)
    err = np.abs(res.sigma - sig) / sig
    print(f"monostatic sigma vs oracle: max rel {err.max():.2e}")
    assert err.max() < 1e-8


def test_monostatic_sweep_mixed_vs_fp64():
    # 1,680-RWG plate, 96 incidences: complex64 Z + tensor-core block GMRES
    # against the plain FP64 path (reference near-field preconditioner, 1 lambda)
    from diffmom_b200 import EFIEDevice, make_plane_wave, monostatic_rcs_sweep
    from diffmom_b200 import compute_farfield, bistatic_rcs, SphGrid
    m = make_rect_plate(0.1, 0.1, 24, 24)
    rwg = build_rwg(m)
    dev = EFIEDevice(m, rwg)
    kv, e0, pol = _waves(K3, 96, 11)
    exc = [make_plane_wave(kv[i], 1.0, pol[i]) for i in range(96)]
    r64 = monostatic_rcs_sweep(m, 3e9, exc, precision="fp64", nf_cutoff_lambda=1.0, gmres_tol=1e-10,
                               device=dev, rwg=rwg, return_currents=True)
    # the fused monostatic kernel agrees with the general far-field path
    for i in (0, 47, 95):
        grid = SphGrid(rhat=(-kv[i] / K3)[None], theta=np.zeros(1), phi=np.zeros(1), w=np.ones(1))
        E = compute_farfield(dev, grid, r64.currents[:, i])
        s_ff = bistatic_rcs(np.asarray(E).reshape(3, -1)[:, :1])[0]
        assert abs(s_ff - r64.sigma[i]) <= 1e-12 * s_ff
    rm = monostatic_rcs_sweep(m, 3e9, exc, precision="mixed", gmres_tol=1e-6, device=dev, rwg=rwg,
                              return_currents=True)
    rel = np.abs(rm.sigma - r64.sigma) / r64.sigma.max()
    cur = np.linalg.norm(rm.currents - r64.currents, axis=0) / np.linalg.norm(r64.currents, axis=0)
    print(f"mixed sweep: {rm.gmres_iters} iterations, {rm.refinements} refinements, true residual "
          f"{rm.true_residual:.2e}; RCS error {rel.max():.2e} of max sigma, current error {cur.max():.2e}")
    assert rm.true_residual <= 1e-6
    assert rel.max() <= 1e-4
    dev.close()


@pytest.mark.parametrize("R", [16, 37, 200])
def test_fp64_zx_many_columns(R):
    # complex128 Z X on the FP64-pipe GEMM (128 x 64 tiles; N = 1,680 and R
    # ragged against them) against numpy's product of the same copied-out Z
    dev = _plate(24)
    Z = dev.assemble(K3, precision="fp64", copy_out=True)
    X = _rand(dev.N, R, 100 + R)
    Y = dev.matvec(X)
    ref = Z @ X
    err = np.linalg.norm(Y - ref) / np.linalg.norm(ref)
    print(f"FP64 Z X, R={R}: {err:.2e}")
    assert err < 1e-13
    dev.close()


def test_fp64_factor_and_sweeps_on_the_fp64_gemm():
    # complete complex128 LDL^T (trailing updates on the FP64-pipe GEMM) and
    # its many-column sweeps: Z^-1 B against numpy's solve
    dev = _plate(24)
    Z = dev.assemble(K3, precision="fp64", copy_out=True)
    dev.build_nearfield(float("inf"), "lu")
    B = _rand(dev.N, 40, 7)
    X = dev.nf_apply(B)
    ref = np.linalg.solve(Z, B)
    err = np.linalg.norm(X - ref) / np.linalg.norm(ref)
    print(f"FP64 factor + sweeps, 40 columns: {err:.2e}")
    assert err < 1e-10
    dev.close()


def test_autotuner_candidates_identical():
    """Every candidate of the online autotuner writes the same bits: the
    complex64 factor (4- or 2-stage update pipelines, persistent lower-tile
    grid) and a batched sweep (256- or 128-wide GEMM tiles, or the persistent
    256-wide grid), pinned one at a time, against the tuned run, with TF32 and
    with BF16 operand pieces; the tuner's report lists what it measured."""
    from diffmom_b200 import tune_report
    dev = _plate(36)  # 3,960 RWG: four 1,024-row sweep blocks, ragged last
    dev.assemble(K3, precision="mixed")
    X = _rand(dev.N, 200, 3)
    for bf in (0, 1):
        dev.set_option("precond_bf16", bf)
        out = {}
        for syrk in (0, 1, 2, 3):
            for gemm in (0, 1, 2, 3):
                if syrk and gemm:
                    continue
                dev.set_option("tune_tc_syrk", syrk)
                dev.set_option("tune_tc_gemm", gemm)
                dev.build_nearfield(math.inf, "lu")
                out[(syrk, gemm)] = dev.nf_apply(X)
        ref = out[(0, 0)]
        for key, Y in out.items():
            assert np.array_equal(Y, ref), (bf, key)
    dev.set_option("precond_bf16", -1)
    dev.set_option("tune_tc_syrk", 0)
    dev.set_option("tune_tc_gemm", 0)
    rep = tune_report()
    print(rep)
    assert "k_tc_gemm" in rep and "k_tc_syrk" in rep
    with pytest.raises(Exception):
        dev.set_option("tune_tc_gemm", 4)
    with pytest.raises(Exception):
        dev.set_option("tune_tc_syrk", 4)
    dev.close()


def test_bf16_preconditioner_operands():
    """BF16 operand pieces (hi + lo, kind::f16 tensor cores) for the complex64
    factor updates and packed sweeps: the preconditioner apply stays within
    1e-3 of the TF32-piece one, and block GMRES with it still meets the FP64
    residual (the criterion) with the same solution."""
    dev = _plate(36)  # 3,960 RWG: four 1,024-row sweep blocks, ragged last
    dev.set_option("precond_bf16", 0)
    dev.assemble(K3, precision="mixed")
    X = _rand(dev.N, 200, 5)
    dev.build_nearfield(math.inf, "lu")
    y32 = dev.nf_apply(X)
    kv, e0, pol = _waves(K3, 128, 4)
    s32, st32 = dev.solve_many(K3, kv, pol, E0s=e0, precision="mixed", preconditioner="lu", cutoff=math.inf,
                               tol=1e-6, precond_side="right")
    dev.set_option("precond_bf16", 1)
    dev.build_nearfield(math.inf, "lu")
    y16 = dev.nf_apply(X)
    err = np.linalg.norm(y16 - y32) / np.linalg.norm(y32)
    s16, st16 = dev.solve_many(K3, kv, pol, E0s=e0, precision="mixed", preconditioner="lu", cutoff=math.inf,
                               tol=1e-6, precond_side="right")
    print(f"BF16 vs TF32 operand pieces: apply {err:.2e}; GMRES iterations {st16.niter} vs {st32.niter}, "
          f"true residual {st16.true_residual:.2e}")
    assert err < 1e-3
    assert st16.solved and st16.true_residual <= 1e-6
    assert np.max(np.abs(s16 - s32) / s32) < 1e-4
    with pytest.raises(Exception):
        dev.set_option("precond_bf16", 2)
    dev.set_option("precond_bf16", -1)
    dev.close()
