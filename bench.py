#!/usr/bin/env python
"""EFIE solves/s on one B200 -- mixed precision, batched and learned paths
against the plain FP64 path on the same GPU.

Headline workload (batched right-hand sides): PEC plate 0.3 x 0.3 m at 3 GHz,
60 x 60 cells -> 7,200 triangles / 10,680 RWG, quad_order 3; 1,024 plane
waves (seed 20260001: theta ~ U[0, 80) deg, phi ~ U[0, 360) deg, half theta-
and half phi-polarised, k_vec = -k r_hat), monostatic RCS of every solution.
A step is the complete job: assemble Z, build the preconditioner, assemble
the 1,024 right-hand sides, GMRES to 1e-6 relative FP64 residual for all of
them, monostatic sigma on the device.  ``value`` = incidences solved per
second (mixed: complex64 Z with FP32 far pairs and FP64 singular terms,
block GMRES preconditioned by the complex64 LDL^T of Z -- tensor-core updates
and sweeps on BF16 hi + lo operand pieces -- with FP64-accurate Krylov
products from int8 residues modulo 13 moduli (Chinese-remainder
recombination), FP64 Arnoldi and the FP64 residual as the criterion).

Variants reported beside it (same timing rules, fewer steps where slow):
  c3_mixed_tf32_refined  the headline with the Krylov product in 3xTF32 and
                  FP64-residual refinement instead of the INT8 product
  c3_mixed_precond_tf32x3 / _tf32x1  the headline with the preconditioner's
                  tensor-core operands as TF32 pieces (3 or 1 products)
  c3_fp64_plain   the same job in plain FP64 (FP64 Z, the reference's
                  near-field LDL^T at 1 lambda, FP64 block GMRES)
  c3_20k_*        the same sweep on a 0.41 m plate (82 x 82 cells, 20,008 RWG)
  c2_*            PEC sphere r = 0.5 lambda, 7,680 RWG, one incidence,
                  FP64 / mixed with the 1-lambda near-field preconditioner
  c4_*            64 impedance-loaded rectangular / circular plates, 0.5-3
                  lambda, 500-6,000 RWG, one incidence each (seed 20260004):
                  mixed on 8 lanes vs plain FP64 one surface at a time;
                  per size-bucket solve times
  c5_*            perturbed ellipsoid (seed 99), 9,720 RWG (c5_17k_*: 17,280),
                  one incidence: FP64 near-field vs mixed + local, plain ring
                  step and learned right preconditioners (the library's
                  default weights, trained on 48 other generated bodies)

``e2e`` times the headline through the public API (monostatic_rcs_sweep)
with host buffers: mesh/RWG/incidence upload and the sigma download inside
the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 (torchrun) every rank solves its own copy (replicas, weak
scaling; the path has no exchange step).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "diffmom.jl_b200"))

C0 = 299792458.0
FREQ = 3e9
LAM = C0 / FREQ
K = 2 * math.pi * FREQ / C0
R_WAVES = 1024
SEED = 20260001
METRIC = "EFIE solves/s (assemble+GMRES to 1e-6) mixed/learned vs plain FP64, 1 B200"
# DRAM bytes per k_oz_gemm launch (13 residue products, R = 1,024) on the
# headline plate, measured with ncu one-pass dram__bytes_read/write.sum
OZ_TRAFFIC_PER_LAUNCH = 12300295168  # mean of the step's two launches: 11.900 + 0.400 GB
WORKLOAD = "pec_plate_0.3m_3GHz_60x60_10680rwg_1024planewaves_monostatic"


PLATE_CELLS = 60


def plate_c3():
    from diffmom_b200 import make_rect_plate, build_rwg
    side = 0.3 * PLATE_CELLS / 60.0   # 60 cells: the 0.3 m, 10,680-RWG plate
    mesh = make_rect_plate(side, side, PLATE_CELLS, PLATE_CELLS)
    return mesh, build_rwg(mesh)


def waves(R=None, seed=SEED):
    """theta ~ U[0, 80) deg, phi ~ U[0, 360) deg; even: theta-pol, odd: phi-pol."""
    R = R_WAVES if R is None else R
    rng = np.random.default_rng(seed)
    th = np.deg2rad(rng.uniform(0.0, 80.0, R))
    ph = np.deg2rad(rng.uniform(0.0, 360.0, R))
    rhat = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], 1)
    tha = np.stack([np.cos(th) * np.cos(ph), np.cos(th) * np.sin(ph), -np.sin(th)], 1)
    pha = np.stack([-np.sin(ph), np.cos(ph), np.zeros(R)], 1)
    pol = np.where((np.arange(R) % 2 == 0)[:, None], tha, pha)
    return np.ascontiguousarray(-K * rhat), np.ones(R), np.ascontiguousarray(pol)


def dist_env():
    from diffmom_b200 import replicas
    return replicas.replica_env()


class Clocks:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        rows = [l.split(",") for l in Path(self.f.name).read_text().splitlines() if l.strip()]
        sm = [float(r[1]) for r in rows if len(r) > 8 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) > 8 and r[2].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) > 8:
                for nm, v in zip(names, r[5:9]):
                    if "Active" in v and "Not" not in v:
                        reasons.add(nm)
        loaded = [s for s in sm if mx and s > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(rows)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
class Runner:
    def __init__(self, local, ws):
        import torch
        self.torch = torch
        self.local, self.ws = local, ws

    def barrier(self):
        from diffmom_b200 import replicas
        replicas.barrier()

    def max_over_ranks(self, x):
        from diffmom_b200 import replicas
        return replicas.max_over_ranks(x, device=f"cuda:{self.local}")

    def timed(self, dev, step, steps, warmup, per_step_units, kernel_timing=False, clocks=False):
        """Device-timed loop on the library's stream: warm-up, barrier + sync,
        events around exactly `steps` steps, barrier + sync, max over ranks."""
        import ctypes as ct
        from diffmom_b200 import _native as nat
        torch = self.torch
        sp = ct.c_void_p()
        dev.ctx.call("dmb_get_stream", ct.byref(sp))
        ext = torch.cuda.ExternalStream(sp.value, device=self.local)
        out = None
        for _ in range(warmup):
            out = step()
        k0 = dev.timings().kernels
        dev.ctx.call("dmb_set_kernel_timing", 1 if kernel_timing else 0)
        clk = Clocks(self.local) if clocks else None
        if clk:
            clk.start()
        self.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        for _ in range(steps):
            out = step()
        e1.record(ext)
        torch.cuda.synchronize()
        self.barrier()
        ms = self.max_over_ranks(e0.elapsed_time(e1))
        tm = dev.timings()
        res = {"ms_per_step": ms / steps, "solves_per_s": self.ws * steps * per_step_units / (ms / 1e3),
               "steps": steps, "warmup": warmup, "launches": tm.kernels - k0,
               "stage_ms_last_step": {"assembly": tm.assembly_ms, "preconditioner": tm.precond_ms,
                                      "rhs": tm.rhs_ms, "gmres": tm.gmres_ms, "total": tm.solve_ms}}
        if clk:
            res["clocks"] = clk.stop()
        if kernel_timing:
            for fam, key in ((0, "kernel_gemm"), (1, "kernel_int8"), (2, "kernel_factor"), (4, "kernel_fp64"),
                             (5, "kernel_assembly")):
                kms, kl, kf = ct.c_double(), ct.c_int64(), ct.c_double()
                dev.ctx.call("dmb_kernel_timing_family", fam, ct.byref(kms), ct.byref(kl), ct.byref(kf))
                res[key] = (kms.value, kl.value, kf.value)
        dev.ctx.call("dmb_set_kernel_timing", 0)
        res["last"] = out
        return res


def measure_fp64_peaks(local):
    """FP64 reference throughput of this GPU, measured with cuBLAS through
    torch (B200 has no FP64 tensor-core kind; MEASURED_PEAKS.json holds bf16
    only): DGEMM 8192^3 (2 n^3 flops) and ZGEMM 4096^3 (8 n^3), best of 5."""
    import torch
    out = {}
    for name, dt, n, fl in (("cublas_dgemm_tflops", torch.float64, 8192, 2.0),
                            ("cublas_zgemm_tflops", torch.complex128, 4096, 8.0)):
        a = torch.randn(n, n, dtype=dt, device=f"cuda:{local}")
        b = torch.randn(n, n, dtype=dt, device=f"cuda:{local}")
        torch.matmul(a, b)
        best = None
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        out[name] = fl * n ** 3 / (best / 1e3) / 1e12
        del a, b
    # dense INT8 reference for the int8 residue products: cuBLASLt through
    # torch._int_mm (int8 x int8 -> int32) at 8192^3, best of 10
    try:
        n = 8192
        a = torch.randint(-127, 128, (n, n), dtype=torch.int8, device=f"cuda:{local}")
        b = torch.randint(-127, 128, (n, n), dtype=torch.int8, device=f"cuda:{local}")
        bt = b.t().contiguous().t()  # column-major right operand, the layout cuBLASLt int8 wants
        torch._int_mm(a, bt)
        best = None
        for _ in range(10):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch._int_mm(a, bt)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        out["cublaslt_int8_pops"] = 2.0 * n ** 3 / (best / 1e3) / 1e15
        del a, b, bt
    except Exception as exc:  # no int8 GEMM in this torch build: report why
        out["cublaslt_int8_unavailable"] = str(exc).splitlines()[0][:160] if str(exc) else type(exc).__name__
    torch.cuda.empty_cache()
    return out


def fp64_roofline(v, peaks):
    """The FP64-pipe GEMM families of a timed FP64 variant: complex flops (8
    per complex MAC) per event-timed launch time, against cuBLAS ZGEMM."""
    out = {"peak_tflops": peaks.get("cublas_zgemm_tflops"), "peak_source": "cuBLAS ZGEMM 4096^3 measured in this run",
           "dgemm_tflops": peaks.get("cublas_dgemm_tflops")}
    for key, name in (("kernel_fp64", "k_zgemm64 (Z X and sweep updates)"),
                      ("kernel_factor", "k_zgemm64 lower (LDL^T trailing updates)")):
        ms, launches, work = v.get(key, (0.0, 0, 0.0))
        if ms > 0:
            ach = (work / 1e12) / (ms / 1e3)
            out[name] = {"achieved_tflops": ach, "launches": launches, "kernel_ms_total": ms,
                         "frac_of_cublas_zgemm": ach / out["peak_tflops"] if out["peak_tflops"] else None}
    return out


def copy_currents(dev, N):
    from diffmom_b200 import _native as nat
    I = np.empty((N, R_WAVES), dtype=np.complex128, order="F")
    dev.ctx.call("dmb_copy_solution", nat.dptr(I))
    return I


def solve_params(nat, k, precision, precond, cutoff, side=0, maxiter=300, kvec=(0.0, 0.0, -1.0),
                 pol=(1.0, 0.0, 0.0)):
    p = nat.SolveParams()
    p.k, p.eta0, p.cutoff, p.tol = k, 376.730313668, cutoff, 1e-6
    p.quad_order, p.precision, p.precond_kind, p.precond_side, p.maxiter = 3, precision, precond, side, maxiter
    p.kvec[:] = [kvec[0] * k, kvec[1] * k, kvec[2] * k]
    p.pol[:] = list(pol)
    p.E0 = 1.0
    return p


def run_ours(args):
    import torch
    from diffmom_b200 import (EFIEDevice, make_plane_wave, monostatic_rcs_sweep, make_icosphere,
                              make_perturbed_ellipsoid, build_rwg)
    from diffmom_b200 import _native as nat

    ws, rank, local = dist_env()
    from diffmom_b200 import replicas
    torch.cuda.set_device(local)
    replicas.init("nccl", timeout_s=300)
    run = Runner(local, ws)
    variants = {}
    fp64_peaks = measure_fp64_peaks(local)
    gpu_results = {}   # variant -> (currents N x R, sigma R) for the oracle comparison
    c2_results = {}    # C2 variant -> (Z, currents, 181-point far field)
    only = set(args.only.split(",")) if args.only else None

    def want(name):
        return only is None or name in only

    # ---- headline: C3 batched sweep --------------------------------------
    # a sweep of ws x 1,024 incidences, one disjoint share of 1,024 per rank
    # (weak scaling; at one GPU the share is the whole 1,024-incidence job)
    mesh, rwg = plate_c3()
    N = rwg.nedges
    start, count = replicas.shard(ws * R_WAVES, ws, rank)
    assert count == R_WAVES and start % R_WAVES == 0
    kv, e0, pol = waves(R_WAVES, seed=SEED + start // R_WAVES)
    dev = EFIEDevice(mesh, rwg, device=local)
    if args.int8_tile:
        dev.set_option("tune_int8_tile", args.int8_tile)
    sig = np.empty(R_WAVES)

    def c3_step(precision, precond, cutoff, side=1):
        p = solve_params(nat, K, precision, precond, cutoff, side=side, maxiter=200)
        st = nat.GmresStats()

        def step():
            dev.ctx.call("dmb_solve_resident_many", ctypes.byref(p), R_WAVES, nat.dptr(kv), nat.dptr(e0),
                         nat.dptr(pol), nat.dptr(sig), ctypes.byref(st))
            return st.niter, st.true_residual, st.restarts
        return step

    head = None
    sig_mixed = None
    if want("c3_mixed_tf32_refined") and not args.quick:
        dev.set_option("exact_krylov", 0)
        variants["c3_mixed_tf32_refined"] = run.timed(dev, c3_step(nat.PREC_MIXED, nat.PRECOND_NF_LU, math.inf),
                                                      min(args.steps, 3), args.warmup, R_WAVES)
        dev.set_option("exact_krylov", 1)
    if want("c3_mixed_batched"):
        head = run.timed(dev, c3_step(nat.PREC_MIXED, nat.PRECOND_NF_LU, math.inf), args.steps, args.warmup,
                         R_WAVES, kernel_timing=True, clocks=True)
        sig_mixed = sig.copy()
        gpu_results["c3_mixed_batched"] = (copy_currents(dev, N), sig_mixed)
        variants["c3_mixed_batched"] = head
        # every rank's share of sigma to rank 0 (after the timed region)
        sig_all = replicas.gather_to_rank0(sig_mixed, device=f"cuda:{local}")
        if rank == 0:
            head["sweep"] = {"incidences_total": int(sig_all.size), "per_rank": R_WAVES, "ranks": ws,
                             "sigma_all_finite_positive": bool(np.all(np.isfinite(sig_all) & (sig_all > 0))),
                             "sigma_gathered_on_rank0": True}
    for name, terms in (("c3_mixed_precond_tf32x3", 3), ("c3_mixed_precond_tf32x1", 1)):
        if not (want(name) and (not args.quick or (only and name in only))):
            continue
        # the same job with the preconditioner's tensor-core operands as TF32
        # pieces (all three products, or hi x hi only)
        dev.set_option("precond_bf16", 0)
        dev.set_option("precond_tf32_terms", terms)
        v = run.timed(dev, c3_step(nat.PREC_MIXED, nat.PRECOND_NF_LU, math.inf), min(args.steps, 3), args.warmup,
                      R_WAVES)
        dev.set_option("precond_tf32_terms", 3)
        dev.set_option("precond_bf16", -1)
        if sig_mixed is not None:
            v["rcs_rel_err_vs_mixed"] = float(np.max(np.abs(sig_mixed - sig)) / np.max(sig_mixed))
        variants[name] = v
    if want("c3_fp64_plain") and not args.quick:
        v = run.timed(dev, c3_step(nat.PREC_FP64, nat.PRECOND_NF_LU, 1.0 * LAM), 1, 1, R_WAVES)
        if sig_mixed is not None:
            v["rcs_rel_err_vs_mixed"] = float(np.max(np.abs(sig_mixed - sig) / sig))
        gpu_results["c3_fp64_plain"] = (copy_currents(dev, N), sig.copy())
        variants["c3_fp64_plain"] = v
    if want("c3_fp64_full_factor") and not args.quick:
        # precision alone: the headline's algorithm (complete LDL^T of Z, right
        # preconditioning, block GMRES) with FP64 Z, factor, sweeps and products
        v = run.timed(dev, c3_step(nat.PREC_FP64, nat.PRECOND_NF_LU, math.inf), min(args.steps, 3), 1, R_WAVES,
                      kernel_timing=True)
        gpu_results["c3_fp64_full_factor"] = (copy_currents(dev, N), sig.copy())
        v["roofline_fp64"] = fp64_roofline(v, fp64_peaks)
        variants["c3_fp64_full_factor"] = v

    # e2e through the public API (host buffers in, sigma out)
    e2e = None
    if head is not None and not args.skip_e2e:
        exc = [make_plane_wave(kv[i], e0[i], pol[i]) for i in range(R_WAVES)]

        def e2e_step():
            dev.ctx.call("dmb_mesh_upload", nat.dptr(mesh.xyz), nat.lptr(mesh.tri), mesh.nvertices,
                         mesh.ntriangles)
            tp, tm, vp, vm, ln, ap, am = dev._arrs
            dev.ctx.call("dmb_rwg_upload", N, nat.lptr(tp), nat.lptr(tm), nat.lptr(dev._evert),
                         nat.lptr(vp), nat.lptr(vm), nat.dptr(ln), nat.dptr(ap), nat.dptr(am))
            r = monostatic_rcs_sweep(mesh, FREQ, exc, precision="mixed", gmres_tol=1e-6, device=dev, rwg=rwg)
            return r.gmres_iters, r.true_residual
        e = run.timed(dev, e2e_step, args.steps, max(1, args.warmup // 2), R_WAVES)
        h2d = (mesh.xyz.nbytes + mesh.tri.nbytes + rwg.evert.nbytes + 7 * 8 * N + 7 * 8 * R_WAVES)
        e2e = {"value": e["solves_per_s"], "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(8 * R_WAVES),
               "api": "diffmom_b200.monostatic_rcs_sweep(precision=mixed) incl. mesh/RWG upload"}
    dev.close()

    # the same sweep at 20,008 RWG (0.41 m plate, 82 x 82 cells, same cell size)
    if want("c3_20k_mixed_batched") and not args.quick and PLATE_CELLS == 60:
        from diffmom_b200 import make_rect_plate as _plate
        m20 = _plate(0.41, 0.41, 82, 82)
        r20 = build_rwg(m20)
        dev20 = EFIEDevice(m20, r20, device=local)
        sig20 = np.empty(R_WAVES)
        p20 = solve_params(nat, K, nat.PREC_MIXED, nat.PRECOND_NF_LU, math.inf, side=1, maxiter=200)
        st20 = nat.GmresStats()

        def step20():
            dev20.ctx.call("dmb_solve_resident_many", ctypes.byref(p20), R_WAVES, nat.dptr(kv), nat.dptr(e0),
                           nat.dptr(pol), nat.dptr(sig20), ctypes.byref(st20))
            return st20.niter, st20.true_residual, st20.restarts
        v20 = run.timed(dev20, step20, 1, 1, R_WAVES)
        v20["N_rwg"] = r20.nedges
        variants["c3_20k_mixed_batched"] = v20
        dev20.close()

    # ---- one incidence on the C3 plate: the reference's H-matrix (ACA) path
    # of solve_scattering (10k < N <= 50k) beside the dense single-RHS path
    if not args.quick and any(want(n) for n in ("plate_1wave_aca", "plate_1wave_dense_mixed")):
        sdev = None
        try:
            hbm_peak = measured_peaks()[0]
            sdev = EFIEDevice(mesh, rwg, device=local)
            v1 = np.ascontiguousarray(sdev.plane_wave_rhs(np.array([[0.0, 0.0, -K]]), [1.0],
                                                          np.array([[1.0, 0.0, 0.0]]))[:, 0])
            x1 = np.empty_like(v1)
            st1 = nat.GmresStats()
            info = nat.AcaInfo()
            if want("plate_1wave_aca"):
                def aca_step():
                    # build_aca_operator defaults of solve_scattering (leaf 64, eta 1.5,
                    # tol 1e-6, rank 50), near-field LU of its dense blocks (complex64),
                    # GMRES to 1e-6
                    sdev.ctx.call("dmb_aca_build", K, 376.730313668, 3, 64, 1.5, 1e-6, 50, 2_000_000, 4_000_000_000,
                                  ctypes.byref(info))
                    sdev.ctx.call("dmb_aca_nf_build", nat.PRECOND_NF_LU, nat.PREC_MIXED, None)
                    sdev.ctx._check(sdev.ctx.lib.dmb_gmres(sdev.ctx.h, nat.dptr(v1), nat.dptr(x1), 1, 1e-6, 300,
                                                           nat.PRECOND_NF_LU, nat.SIDE_LEFT, 1, ctypes.byref(st1)))
                    return st1.niter, st1.true_residual, st1.restarts
                va = run.timed(sdev, aca_step, min(args.steps, 3), 1, 1)
                va["aca"] = {f: getattr(info, f) for f, _ in nat.AcaInfo._fields_}
                va["aca"]["stored_fraction_of_dense"] = info.entries_stored / float(N) ** 2
                # H-matrix product alone: event-timed inside the library (family 3)
                xr = np.ascontiguousarray(np.random.default_rng(1).standard_normal(N) + 0j)
                yr = np.empty_like(xr)
                sdev.ctx.call("dmb_aca_matvec", nat.dptr(xr), nat.dptr(yr), 1, 0)
                sdev.ctx.call("dmb_set_kernel_timing", 1)
                for _ in range(20):
                    sdev.ctx.call("dmb_aca_matvec", nat.dptr(xr), nat.dptr(yr), 1, 0)
                kms, kl, kw = ctypes.c_double(), ctypes.c_int64(), ctypes.c_double()
                sdev.ctx.call("dmb_kernel_timing_family", 3, ctypes.byref(kms), ctypes.byref(kl), ctypes.byref(kw))
                sdev.ctx.call("dmb_set_kernel_timing", 0)
                gbs = (kw.value / 1e9) / (kms.value / 1e3) if kms.value > 0 else None
                va["product"] = {"ms": kms.value / max(kl.value, 1), "launch_groups": kl.value,
                                 "bytes_per_product": kw.value / max(kl.value, 1), "achieved_gbs": gbs,
                                 "frac_of_measured_hbm": (gbs / hbm_peak) if gbs else None}
                variants["plate_1wave_aca"] = va
            if want("plate_1wave_dense_mixed"):
                p1 = solve_params(nat, K, nat.PREC_MIXED, nat.PRECOND_NF_LU, math.inf, side=1, maxiter=300)

                def dense_step():
                    sdev.ctx.call("dmb_solve_resident", ctypes.byref(p1), ctypes.byref(st1))
                    return st1.niter, st1.true_residual, st1.restarts
                variants["plate_1wave_dense_mixed"] = run.timed(sdev, dense_step, min(args.steps, 3), 1, 1)
            sdev.close()
        except Exception as e:  # optional variants: the headline line still prints
            for name in ("plate_1wave_aca", "plate_1wave_dense_mixed"):
                if want(name) and name not in variants:
                    variants[name] = {"error": f"{type(e).__name__}: {e}"[:300]}
            if sdev is not None:
                sdev.close()

    # ---- C4 uneven batch of 64 impedance-loaded surfaces -------------------
    if not args.quick and any(want(n) for n in ("c4_batch64_mixed", "c4_batch64_fp64", "c4_batch64_fp64_1lane")):
        from diffmom_b200 import SurfaceBatch
        from diffmom_b200.workloads import impedance_surface_batch
        surf = impedance_surface_batch(64)
        for name, prec, lanes in (("c4_batch64_mixed", "mixed", 8), ("c4_batch64_fp64", "fp64", 8),
                                  ("c4_batch64_fp64_1lane", "fp64", 1)):
            if not want(name):
                continue
            batch = SurfaceBatch(lanes, device=local)
            reps = min(args.steps, 3) if prec == "mixed" else 1
            for _ in range(1 if prec == "fp64" else args.warmup):
                batch.solve(surf, K, precision=prec)
            run.barrier()
            dms, last = [], None
            for _ in range(reps):
                last = batch.solve(surf, K, precision=prec)
                dms.append(last.device_ms)
            batch.close()
            ms = run.max_over_ranks(float(np.mean(dms)))
            buckets = {}
            for lo, hi in ((500, 1500), (1500, 3000), (3000, 4500), (4500, 6500)):
                sel = (last.N >= lo) & (last.N < hi)
                if sel.any():
                    buckets[f"N{lo}-{hi}"] = {"surfaces": int(sel.sum()),
                                             "solve_ms_mean": float(last.solve_ms[sel].mean()),
                                             "latency_ms_max": float(last.latency_ms[sel].max()),
                                             "surfaces_per_s_alone": float(1e3 / last.solve_ms[sel].mean())}
            variants[name] = {"ms_per_step": ms, "solves_per_s": ws * 64 / (ms / 1e3), "steps": reps,
                              "warmup": 1 if prec == "fp64" else args.warmup, "launches": None, "lanes": lanes,
                              "last": (int(last.gmres_iters.max()), float(last.true_residual.max())),
                              "buckets": buckets, "sum_N2": float(np.sum(last.N.astype(float) ** 2)),
                              "assembly_ms_all_surfaces": float(last.assembly_ms),
                              "assembly": "every surface's Z by one far-pair tile launch (task list of all "
                                          "surfaces' RWG tile pairs, largest first) + one near-values and one "
                                          "near-sums launch"}

    # ---- C2 sphere, one incidence -----------------------------------------
    if not args.quick and (want("c2_fp64_nf_lu") or want("c2_mixed_nf_lu")):
        sph, srwg = c2_sphere()
        sdev = EFIEDevice(sph, srwg, device=local)
        for name, prec in (("c2_fp64_nf_lu", nat.PREC_FP64), ("c2_mixed_nf_lu", nat.PREC_MIXED)):
            if not want(name):
                continue
            p = solve_params(nat, K, prec, nat.PRECOND_NF_LU, 1.0 * LAM)
            st = nat.GmresStats()

            def step(p=p, st=st):
                sdev.ctx.call("dmb_solve_resident", ctypes.byref(p), ctypes.byref(st))
                return st.niter, st.true_residual
            variants[name] = run.timed(sdev, step, min(args.steps, 5), args.warmup, 1)
            # results for the evaluation against the oracle (untimed): currents
            # of the timed solve, 181-point phi = 0 bistatic far field, and Z
            I1 = np.empty(srwg.nedges, dtype=np.complex128)
            sdev.ctx.call("dmb_copy_solution", nat.dptr(I1))
            E1 = sdev.farfield(c2_grid().rhat, I1, k=K)
            Zc = sdev.assemble(K, precision="fp64" if prec == nat.PREC_FP64 else "mixed", copy_out=True)
            c2_results[name] = (Zc, I1, E1)
        if want("c2_fp64_nf_lu"):
            # the FP64 path solved to 1e-10 (untimed): the currents / RCS parity level
            p = solve_params(nat, K, nat.PREC_FP64, nat.PRECOND_NF_LU, 1.0 * LAM)
            p.tol = 1e-10
            st = nat.GmresStats()
            sdev.ctx.call("dmb_solve_resident", ctypes.byref(p), ctypes.byref(st))
            I1 = np.empty(srwg.nedges, dtype=np.complex128)
            sdev.ctx.call("dmb_copy_solution", nat.dptr(I1))
            c2_results["c2_fp64_nf_lu_tol1e-10"] = (c2_results["c2_fp64_nf_lu"][0], I1,
                                                    sdev.farfield(c2_grid().rhat, I1, k=K))
        sdev.close()

    # ---- C5 perturbed ellipsoid, learned right preconditioner -------------
    if not args.quick and any(want(n) for n in ("c5_fp64_nf_lu", "c5_mixed_nf_lu", "c5_mixed_learned",
                                                 "c5_mixed_local")):
        r_nb = 0.2 * LAM
        from diffmom_b200.learned import DEFAULT_WEIGHTS
        body = make_perturbed_ellipsoid(LAM, 99, frequency=18)
        brwg = build_rwg(body)
        tdev = EFIEDevice(body, brwg, device=local)
        # the library's default weights: trained on the GPU over 48 generated
        # bodies (python -m diffmom_b200.learned), none of them this one
        net_note = "default weights (48 generated training bodies)"
        if DEFAULT_WEIGHTS.exists():
            tdev.load_network(DEFAULT_WEIGHTS)
        else:
            from diffmom_b200.learned import train_learned_network, training_bodies
            rep = train_learned_network(tdev, training_bodies(16))
            net_note = f"trained here (untimed) on 16 generated bodies, {rep.gpu_s:.1f} s"
            tdev.upload(body, brwg)
        for freq_f, tag in ((18, "c5"), (24, "c5_17k")):
            if freq_f != 18:
                body = make_perturbed_ellipsoid(LAM, 99, frequency=freq_f)
                brwg = build_rwg(body)
                tdev.upload(body, brwg)
            cases = [("c5_fp64_nf_lu", nat.PREC_FP64, nat.PRECOND_NF_LU, 1.0 * LAM, 0),
                     ("c5_mixed_nf_lu", nat.PREC_MIXED, nat.PRECOND_NF_LU, 1.0 * LAM, 0)] if tag == "c5" else []
            cases += [(f"{tag}_mixed_local", nat.PREC_MIXED, nat.PRECOND_LOCAL_INV, r_nb, 1),
                      (f"{tag}_mixed_ring", nat.PREC_MIXED, nat.PRECOND_RING, r_nb, 1),
                      (f"{tag}_mixed_learned", nat.PREC_MIXED, nat.PRECOND_LEARNED, r_nb, 1)]
            for name, prec, pc, cut, side in cases:
                if not want(name) and not want(name.replace("c5_17k", "c5")):
                    continue
                st = nat.GmresStats()
                p = solve_params(nat, K, prec, pc, cut, side=side, maxiter=600)

                def step(p=p, st=st):
                    tdev.ctx.call("dmb_solve_resident", ctypes.byref(p), ctypes.byref(st))
                    return st.niter, st.true_residual
                variants[name] = run.timed(tdev, step, min(args.steps, 5), args.warmup, 1)
                variants[name]["N_rwg"] = brwg.nedges
                variants[name]["network"] = net_note
        tdev.close()

    line = make_line(args, ws, N, mesh, head, variants, e2e, fp64_peaks) if rank == 0 else None
    if rank == 0:
        line["fp64_peaks_measured"] = fp64_peaks
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        # the complete job on the host cores: the CPU baseline, and the oracle
        # every GPU result of the headline workload is checked against
        job = cpu_c3_job(kv, e0, pol, mesh, rwg)
        line["cpu_baseline"] = cpu_baseline(job)
        line["parity_vs_oracle"] = {name: parity_vs_oracle(job, cur, sg) for name, (cur, sg) in gpu_results.items()}
        del job
        if c2_results:
            line["c2_eval"] = c2_evaluation(c2_results)
    if rank == 0:
        print(json.dumps(line), flush=True)
    replicas.finalize()


def clean(v):
    out = {k: x for k, x in v.items()
           if k not in ("kernel_gemm", "kernel_int8", "kernel_factor", "kernel_fp64", "launches", "last", "clocks")}
    last = v.get("last")
    if last is not None:
        out["gmres_iters"] = int(last[0])
        out["true_residual"] = float(last[1])
        if len(last) > 2:
            out["refinement_cycles"] = int(last[2])
    if v.get("launches") is not None:
        out["kernels_per_step"] = v["launches"] / v["steps"]
    return out


def make_line(args, ws, N, mesh, head, variants, e2e, fp64_peaks=None):
    hbm, bf16, src = measured_peaks()
    base = variants.get("c3_fp64_plain")
    speed = {}
    if head is not None and base is not None:
        speed["c3_mixed_batched_vs_c3_fp64_plain"] = head["solves_per_s"] / base["solves_per_s"]
    full = variants.get("c3_fp64_full_factor")
    if head is not None and full is not None:
        # the total gain splits into precision (same algorithm in FP64) and
        # algorithm (complete factor vs the reference's 1-lambda near field, FP64)
        speed["precision_gain_c3_mixed_batched_vs_c3_fp64_full_factor"] = head["solves_per_s"] / full["solves_per_s"]
        if base is not None:
            speed["algorithm_gain_c3_fp64_full_factor_vs_c3_fp64_plain"] = full["solves_per_s"] / base["solves_per_s"]
    for a, b in (("c3_mixed_batched", "c3_mixed_precond_tf32x3"), ("c4_batch64_mixed", "c4_batch64_fp64"), ("c4_batch64_fp64", "c4_batch64_fp64_1lane"),
                 ("c2_mixed_nf_lu", "c2_fp64_nf_lu"), ("c5_mixed_learned", "c5_fp64_nf_lu"),
                 ("c5_mixed_nf_lu", "c5_fp64_nf_lu"), ("c5_mixed_local", "c5_fp64_nf_lu"),
                 ("c5_mixed_learned", "c5_mixed_local"), ("c5_mixed_learned", "c5_mixed_ring"),
                 ("c5_17k_mixed_learned", "c5_17k_mixed_local"), ("c5_17k_mixed_learned", "c5_17k_mixed_ring"),
                 ("plate_1wave_dense_mixed", "plate_1wave_aca")):
        if "solves_per_s" in variants.get(a, {}) and "solves_per_s" in variants.get(b, {}):
            speed[f"{a}_vs_{b}"] = variants[a]["solves_per_s"] / variants[b]["solves_per_s"]
    line = {
        "metric": METRIC,
        "value": head["solves_per_s"] if head else None,
        "unit": "solves/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": head["ms_per_step"] if head else None,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c64 Z (fp32 far pairs, fp64 singular terms), BF16x3 (hi+lo) tensor-core factor updates/sweeps, int8-residue (CRT) FP64-accurate Z X, fp64 Arnoldi",
        "data": "synthetic plate mesh and seeded incidences (seed 20260001)",
        "config": config_dict(N, mesh.ntriangles, ws),
        "variants": {k: clean(v) for k, v in variants.items()},
        "speedups": speed,
        "e2e": e2e,
        "gpu_launches": int(head["launches"]) if head else 0,
    }
    if head is not None:
        # dominant kernel: k_oz_gemm, the Z X products of block GMRES (the
        # Krylov products, R columns each; the true residual is formed from them)
        ims, il, iw = head["kernel_int8"]
        i8_meas = (fp64_peaks or {}).get("cublaslt_int8_pops")
        i8_peak = i8_meas or 4.5
        i8_src = ("measured in this run: cuBLASLt int8 GEMM (torch._int_mm) 8192^3, best of 10" if i8_meas else
                  "nominal dense INT8 (no int8 GEMM measurement available)")
        if il > 0:
            alg = il * 8.0 * N * N * R_WAVES  # 8 flops per complex MAC, counted once
            achieved = (alg / 1e12) / (ims / 1e3)
            prods = iw / (il * 8.0 * N * N * R_WAVES)  # int8 products per launch
            line["roofline"] = {
                "kernel": "k_oz_gemm (Z X with R = %d columns: FP64-accurate complex GEMM from int8 residue "
                          "products on tcgen05 kind::i8, CRT recombination)" % R_WAVES,
                "bound": "tensor", "achieved": achieved, "peak": bf16, "unit": "TFLOP/s",
                "frac": achieved / bf16 if bf16 else None,
                "traffic": OZ_TRAFFIC_PER_LAUNCH if PLATE_CELLS == 60 and R_WAVES == 1024 else None,
                "traffic_note": "DRAM bytes per launch (ncu one-pass dram__bytes metrics of the step's two "
                                "13-product launches on the headline plate)",
                "peak_source": f"{src} dense bf16 (MEASURED_PEAKS.json); algorithmic flops 8 N^2 R per launch "
                               "(complex MAC = 8 real flops, counted once however the product is executed)",
                "launches_timed": il, "kernel_ms_total": ims,
                "kernel_share_of_step": ims / (head["ms_per_step"] * head["steps"]),
                "executed_int8": {"achieved_pops": (iw / 1e15) / (ims / 1e3), "peak_pops": i8_peak,
                                  "frac": (iw / 1e15) / (ims / 1e3) / i8_peak,
                                  "peak_source": i8_src, "nominal_dense_pops": 4.5,
                                  "note": "%.0f int8 products (one per modulus) of the real-stacked "
                                          "(2N x 2N) x (2N x R) system per launch (FP64-accurate Krylov "
                                          "products; the true residual comes from them)" % prods}}
        fams = {"k_tc_gemm (triangular-sweep GEMMs)": head["kernel_gemm"],
                "k_tc_syrk + k_tc_pack (factorisation trailing updates)": head["kernel_factor"]}
        line["roofline_tc"] = {
            "kernel": "tcgen05 complex GEMMs of the preconditioner (build and apply), BF16 hi + lo operand pieces",
            "bound": "tensor", "peak": bf16, "unit": "TFLOP/s",
            "peak_source": f"{src} dense bf16 (MEASURED_PEAKS.json); algorithmic complex flops (8 per complex "
                           "MAC), the three-product split executes 3x that at the bf16 rate",
            "note": "factor updates run on two side streams beside the panel chain: their event times "
                    "include time shared with concurrent kernels",
            "families": {name: {"achieved": (f[2] / 1e12) / (f[0] / 1e3) if f[0] > 0 else 0.0,
                                "frac": (f[2] / 1e12) / (f[0] / 1e3) / bf16 if f[0] > 0 and bf16 else None,
                                "launches_timed": f[1], "kernel_ms_total": f[0],
                                "kernel_share_of_step": f[0] / (head["ms_per_step"] * head["steps"])}
                         for name, f in fams.items()}}
        line["roofline_assembly"] = assembly_roofline(head, full, hbm, N, mesh.ntriangles,
                                                      (fp64_peaks or {}).get("cublas_dgemm_tflops"))
        line["clocks"] = head.get("clocks")
    return line


def assembly_roofline(head, full, hbm, N, Nt, fp64_peak):
    """The far-pair tile kernel of the assembly (k_far_tile), per event-timed
    launch: algorithmic flops on the pinned triangle-pair convention -- 600
    flops per ordered far triangle pair, P_far = Nt^2 - Nt - 2N (9 quadrature
    pairs x (14 kernel + 32 moment flops) + 186 for the 3 x 3 combination) --
    against the measured FP64 peak (cuBLAS DGEMM of this run) for the FP64
    flavour, and the bytes of Z it writes (16 N^2 complex128, 8 N^2 complex64;
    it reads only L2-resident triangle panels) against the measured copy
    bandwidth.  Pipe utilisation comes from the ncu capture (profiles/)."""
    p_far = float(Nt) * Nt - Nt - 2.0 * N
    flops = 600.0 * p_far
    out = {"kernel": "k_far_tile (far triangle pairs written straight into Z by RWG tiles)",
           "bound": "fp64 pipe (fp32 pipe for the mixed flavour)", "unit": "TFLOP/s",
           "algorithmic_flops_per_launch": flops, "peak_fp64": fp64_peak, "peak_hbm_gbs": hbm,
           "note": "600 flops per ordered far triangle pair (pinned convention); Z written once"}
    for key, v, esz in (("mixed_c64", head, 8.0), ("fp64_c128", full, 16.0)):
        if not v or "kernel_assembly" not in v:
            continue
        ms, launches, work = v["kernel_assembly"]
        if launches > 0 and ms > 0:
            per = ms / launches
            ach = (flops / 1e12) / (per / 1e3)
            out[key] = {"launches_timed": launches, "ms_per_launch": per, "achieved_tflops": ach,
                        "frac_fp64_peak": ach / fp64_peak if (fp64_peak and esz == 16.0) else None,
                        "z_write_gbs": (esz * N * N / 1e9) / (per / 1e3),
                        "frac_hbm": (esz * N * N / 1e9) / (per / 1e3) / hbm if hbm else None}
    return out


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (C restatement of the reference algorithm, OpenMP)
# ---------------------------------------------------------------------------
def cpu_c3_job(kv, e0, pol, mesh=None, rwg=None):
    """One complete headline job on the host cores, every stage timed, nothing
    extrapolated: (a) assembly of the whole complex128 Z by the oracle, the C
    restatement of the reference's assemble_Z_efie (per-RWG-pair loop over
    triangle pairs, EFIE.jl:699-753, OpenMP rows, symmetric fill); (b) the
    1,024 plane-wave right-hand sides (assemble_plane_wave, Excitation.jl:
    2866-2896, one incidence per host thread); (c) LAPACK zgetrf of that Z (the
    LU of solve_forward(:direct), Solve.jl:1124-1198 -- the reference's
    near-field GMRES would run 15-30 dense Z x products per incidence instead);
    (d) zgetrs for all incidences at once; (e) monostatic sigma from the
    oracle's radiation vectors (FarField.jl:425-582, Diagnostics.jl:460-517).
    Returns the stage times, the currents and sigma."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc
    import scipy.linalg as sla
    from concurrent.futures import ThreadPoolExecutor
    cores = os.cpu_count() or 1
    omp = min(cores, orc.max_threads())
    if mesh is None:
        mesh, rwg = plate_c3()
    R = len(e0)
    t = {}
    t0 = time.perf_counter()
    c = orc.OracleCache(mesh, rwg, 3)
    Z = c.assemble_z(K, nthreads=omp)
    t1 = time.perf_counter()
    with ThreadPoolExecutor(cores) as ex:
        cols = list(ex.map(lambda i: c.plane_wave_rhs(kv[i], e0[i], pol[i]), range(R)))
    V = np.asfortranarray(np.stack(cols, 1))
    t2 = time.perf_counter()
    lu = sla.lu_factor(Z, overwrite_a=True, check_finite=False)
    t3 = time.perf_counter()
    I = sla.lu_solve(lu, V, check_finite=False)
    t4 = time.perf_counter()
    sig = np.empty(R)
    for a in range(0, R, 128):
        b = min(R, a + 128)
        G = c.radiation_vectors(-kv[a:b] / K, K)            # (3 (b - a)) x N
        E = np.einsum("qcn,nq->qc", G.reshape(b - a, 3, -1), I[:, a:b])
        sig[a:b] = 4 * math.pi * np.sum(np.abs(E) ** 2, axis=1) / np.abs(e0[a:b]) ** 2
    t5 = time.perf_counter()
    del lu, Z
    t.update(assembly_s=t1 - t0, rhs_s=t2 - t1, factor_s=t3 - t2, solves_s=t4 - t3, rcs_s=t5 - t4,
             total_s=t5 - t0)
    return {"times": t, "currents": I, "sigma": sig, "cores": cores, "omp_threads": omp, "N": rwg.nedges}


def cpu_job_summary(job):
    t = job["times"]
    return (f"the complete job, timed: oracle assembly of the full {job['N']} x {job['N']} complex128 Z "
            f"({job['omp_threads']} OpenMP threads) {t['assembly_s']:.1f} s, {R_WAVES} plane-wave RHS "
            f"{t['rhs_s']:.1f} s, LAPACK zgetrf {t['factor_s']:.1f} s, zgetrs of all incidences "
            f"{t['solves_s']:.1f} s, monostatic sigma {t['rcs_s']:.1f} s")


def cpu_baseline(job=None):
    """The headline job on the host cores (rank 0, N = 1): one complete run of
    cpu_c3_job (the oracle port of the reference algorithm + LAPACK)."""
    if job is None:
        kv, e0, pol = waves()
        job = cpu_c3_job(kv, e0, pol)
    t = job["times"]
    return {"value": R_WAVES / t["total_s"], "unit": "solves/s", "cores": job["cores"], "kind": "port",
            "sample": cpu_job_summary(job), "stage_s": {k: round(v, 3) for k, v in t.items()}}


def parity_vs_oracle(job, currents, sigma):
    """Per-incidence errors of GPU currents and monostatic sigma against the
    oracle's complete CPU job (LAPACK solve of the oracle's FP64 Z)."""
    Io, so = job["currents"], job["sigma"]
    cur = np.linalg.norm(currents - Io, axis=0) / np.linalg.norm(Io, axis=0)
    sg = np.abs(sigma - so) / so
    return {"incidences": int(len(so)), "current_rel_err_max": float(cur.max()),
            "current_rel_err_median": float(np.median(cur)), "sigma_rel_err_max": float(sg.max()),
            "sigma_rel_err_median": float(np.median(sg)),
            "oracle": "complex128 Z of the C oracle, LAPACK zgetrf/zgetrs, oracle radiation vectors"}


def c2_sphere():
    from diffmom_b200 import make_icosphere, build_rwg
    sph = make_icosphere(0.5 * LAM, 4)
    return sph, build_rwg(sph)


def c2_grid():
    from diffmom_b200 import phi_cut_grid
    return phi_cut_grid(0.0, np.arange(0, 181, 1.0))


def c2_evaluation(results):
    """The C2 sphere (7,680 RWG, x-polarised wave along -z) against the
    oracle: FP64 Z entrywise, mixed Z normwise; currents and the 181-point
    phi = 0 bistatic RCS of every timed variant vs the oracle's LAPACK solve
    of its own Z, and the mixed results vs the FP64 ones; the Mie series as a
    physics check (runtests.jl:5176-5240 thresholds)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc
    import scipy.linalg as sla
    from diffmom_b200 import bistatic_rcs
    sph, srwg = c2_sphere()
    grid = c2_grid()
    c = orc.OracleCache(sph, srwg, 3)
    Zo = c.assemble_z(K, nthreads=min(os.cpu_count() or 1, orc.max_threads()))
    vo = c.plane_wave_rhs([0.0, 0.0, -K], 1.0, [1.0, 0.0, 0.0])
    zmax = np.max(np.abs(Zo))
    out = {"N_rwg": srwg.nedges, "directions": int(len(grid.rhat))}
    big = np.abs(Zo) > 1e-4 * zmax
    for name, (Z, _, _) in results.items():
        d = np.abs(Z - Zo)
        out[name] = {"Z_rel_err_entrywise_max": float(np.max(d[big] / np.abs(Zo[big]))),
                     "Z_rel_err_normwise": float(np.linalg.norm(Z - Zo) / np.linalg.norm(Zo))}
        del d
    Io = sla.solve(Zo, vo, check_finite=False)
    del Zo
    G = c.radiation_vectors(grid.rhat, K)
    so = bistatic_rcs((G @ Io).reshape(-1, 3).T)
    a = float(np.mean(np.linalg.norm(sph.xyz - sph.xyz.mean(axis=0), axis=1)))
    mie = np.array([orc.mie_bistatic_rcs_pec(K, a, [0, 0, -1], [1, 0, 0], d) for d in grid.rhat])
    for name, (_, I, E) in results.items():
        sg = bistatic_rcs(E)
        dB = 10 * np.log10(sg) - 10 * np.log10(mie)
        out[name].update({
            "current_rel_err_vs_oracle": float(np.linalg.norm(I - Io) / np.linalg.norm(Io)),
            "rcs_rel_err_vs_oracle_max": float(np.max(np.abs(sg - so) / so)),
            "rcs_rel_err_vs_oracle_of_max_sigma": float(np.max(np.abs(sg - so)) / so.max()),
            "mie_mae_db": float(np.mean(np.abs(dB))), "mie_max_db": float(np.max(np.abs(dB)))})
    if "c2_fp64_nf_lu" in results and "c2_mixed_nf_lu" in results:
        Z64, I64, E64 = results["c2_fp64_nf_lu"]
        Zm, Im, Em = results["c2_mixed_nf_lu"]
        s64, sm = bistatic_rcs(E64), bistatic_rcs(Em)
        out["mixed_vs_fp64"] = {"Z_rel_err_normwise": float(np.linalg.norm(Zm - Z64) / np.linalg.norm(Z64)),
                                "current_rel_err": float(np.linalg.norm(Im - I64) / np.linalg.norm(I64)),
                                "rcs_rel_err_max": float(np.max(np.abs(sm - s64) / s64))}
    out["oracle"] = "complex128 Z of the C oracle, LAPACK solve, oracle radiation vectors; Mie series (Bohren-Huffman)"
    return out


def config_dict(N, ntri, ws):
    return {"workload": WORKLOAD, "N_rwg": N, "N_tri": ntri, "incidences": R_WAVES,
            "quad_order": 3, "gmres_tol": 1e-6,
            "precond": "complex64 LDL^T of Z (near-field cutoff = inf), right (flexible form)",
            "krylov_product": "FP64-accurate Z X from int8 residues modulo 13 moduli on tcgen05 (kind::i8), CRT recombination",
            "variant": "c3_mixed_batched", "parallelism": f"incidence shards x{ws} (1,024 per GPU, no data-path collective)",
            "l2": "inputs larger than L2 (Z 912 MB complex64; packed factor 2 x 2.8 GB)"}


def run_reference(args):
    """The reference arm: the reference's algorithm on the host cores (the
    oracle port: Julia is absent), one complete headline job per step."""
    ws, rank, local = dist_env()
    if rank != 0:
        return
    kv, e0, pol = waves()
    mesh, rwg = plate_c3()
    times = []
    job = None
    for i in range(args.warmup + args.steps):
        job = cpu_c3_job(kv, e0, pol, mesh, rwg)
        if i >= args.warmup:
            times.append(job["times"]["total_s"])
    ms = 1e3 * float(np.mean(times))
    v = R_WAVES / (ms / 1e3)
    line = {"metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic plate mesh and seeded incidences (seed 20260001)", "impl": "reference",
            "config": config_dict(rwg.nedges, mesh.ntriangles, ws),
            "reference_impl": "oracle port of the reference algorithm (C, OpenMP) + LAPACK (OpenBLAS) on the "
                              "host cores; Julia is not installed",
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": job["cores"], "kind": "port",
                             "sample": cpu_job_summary(job) + f"; mean of {args.steps} timed jobs"},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def assembly_case():
    """One far-pair tile launch per precision on the C2 sphere (tile widths
    pinned, so the autotuner launches nothing else): the ncu capture case."""
    from diffmom_b200 import EFIEDevice
    sph, srwg = c2_sphere()
    dev = EFIEDevice(sph, srwg)
    for prec, w in (("fp64", 32), ("mixed", 64)):
        dev.set_option("far_tile", w)
        dev.assemble(K, precision=prec)
        print(prec, srwg.nedges, "assembly_ms", dev.timings().assembly_ms)
    dev.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--only", default=None, help="comma-separated variants to run (profiling)")
    ap.add_argument("--quick", action="store_true", help="headline only (profiling)")
    ap.add_argument("--skip-e2e", action="store_true", help="omit the e2e leg (profiling)")
    ap.add_argument("--plate-cells", type=int, default=60,
                    help="profiling case: plate of this many cells per side (same cell size)")
    ap.add_argument("--waves", type=int, default=1024, help="profiling case: number of incidences")
    ap.add_argument("--int8-tile", type=int, default=0, choices=[0, 1, 2],
                    help="profiling: pin the int8 product's tile on the headline device (1: one SM, 2: CTA pair)")
    ap.add_argument("--assembly-case", action="store_true",
                    help="profiling case: assemble the 7,680-RWG sphere once in FP64 (tile width 32) and once "
                         "in mixed precision (tile width 64), print the times and exit")
    args = ap.parse_args()
    if args.assembly_case:
        assembly_case()
        return
    global PLATE_CELLS, R_WAVES, WORKLOAD
    if args.plate_cells != 60 or args.waves != 1024:
        PLATE_CELLS, R_WAVES = args.plate_cells, args.waves
        WORKLOAD = f"profiling case: plate {PLATE_CELLS}x{PLATE_CELLS} cells, {R_WAVES} plane waves"
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
