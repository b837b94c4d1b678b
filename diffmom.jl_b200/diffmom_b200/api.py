"""Host-side mirror of DiffMoM.jl's public API for the dense EFIE path.

Same names, argument meaning and error behaviour as the Julia functions; the
numerical work runs in libdiffmom_b200.so on the GPU.

* ``EFIEDevice``            -- one device context bound to (mesh, rwg): the
                               resident cache, Z and preconditioner.
* ``assemble_Z_efie``       -- src/assembly/EFIE.jl:699-753
* ``matrixfree_efie_operator`` -- src/assembly/EFIE.jl:975-1000
* ``make_plane_wave`` / ``assemble_excitation`` / ``assemble_plane_wave`` /
  ``assemble_multiple_excitations`` -- src/assembly/Excitation.jl
* ``precompute_patch_mass`` / ``assemble_full_Z`` (per-triangle impedance)
  -- src/assembly/Impedance.jl:304-408, src/solver/Solve.jl:1412-1449
* ``build_nearfield_preconditioner`` / ``NearFieldOperator`` --
  src/solver/NearFieldPreconditioner.jl:670-1054
* ``solve_gmres`` -- src/solver/IterativeSolve.jl:341-392
* ``solve_forward`` -- src/solver/Solve.jl:1342-1382
* ``solve_scattering`` / ``ScatteringResult`` -- src/Workflow.jl:67-317
* ``make_sph_grid`` / ``radiation_vectors``-free ``compute_farfield`` /
  ``bistatic_rcs`` / ``backscatter_rcs`` -- FarField.jl, Diagnostics.jl
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import _native as nat
from .mesh import TriMesh, mesh_edge_max
from .rwg import RWGData, build_rwg

C0_DEFAULT = 299792458.0
ETA0_DEFAULT = 376.730313668

_PRECISIONS = {"fp64": nat.PREC_FP64, "mixed": nat.PREC_MIXED}
NET_MAGIC = b"DMBNET1\0"


def _frequency_to_wavenumber(freq_hz: float, c0: float = C0_DEFAULT) -> float:
    """Excitation.jl:358-372: k = 2 pi f / c0."""
    w = 2 * math.pi * float(freq_hz)
    k = w / c0 if math.isfinite(w) else float(freq_hz) * (2 * math.pi / c0)
    if not (math.isfinite(k) and k > 0):
        raise ValueError("frequency is outside the representable wavenumber range")
    return k


# ---------------------------------------------------------------------------
# device-bound system
# ---------------------------------------------------------------------------
class EFIEDevice:
    """Device context holding one mesh + RWG basis (and then Z, preconditioner)."""

    def __init__(self, mesh: TriMesh, rwg: RWGData, device: int = 0):
        self.ctx = nat.Context(device)
        self.upload(mesh, rwg)

    def upload(self, mesh: TriMesh, rwg: RWGData) -> None:
        """(Re)bind the context to a mesh and basis; trained network weights stay."""
        if rwg.mesh is not mesh:
            raise ValueError("RWG data was built for a different mesh")
        self.mesh = mesh
        self.rwg = rwg
        self.N = rwg.nedges
        self.ctx.call("dmb_mesh_upload", nat.dptr(mesh.xyz), nat.lptr(mesh.tri),
                      mesh.nvertices, mesh.ntriangles)
        self._evert = np.ascontiguousarray(rwg.evert, dtype=np.int64)
        self._arrs = [np.ascontiguousarray(a, dtype=t) for a, t in (
            (rwg.tplus, np.int64), (rwg.tminus, np.int64), (rwg.vplus_opp, np.int64),
            (rwg.vminus_opp, np.int64), (rwg.len, np.float64), (rwg.area_plus, np.float64),
            (rwg.area_minus, np.float64))]
        tp, tm, vp, vm, ln, ap, am = self._arrs
        self.ctx.call("dmb_rwg_upload", rwg.nedges, nat.lptr(tp), nat.lptr(tm),
                      nat.lptr(self._evert), nat.lptr(vp), nat.lptr(vm), nat.dptr(ln),
                      nat.dptr(ap), nat.dptr(am))
        self.k = None
        self.precision = None
        self.quad_order = 3
        self.preconditioner = None

    def set_option(self, name: str, value: int) -> None:
        """Implementation switches: "tensor_cores" (0/1) for the complex64
        factorisation update, "tc_min_rhs" (>= 1) for the right-hand-side count
        from which Z X and the batched near-field solves use the tensor cores,
        "far_tile" (0 = autotuned; FP64 16/32, mixed 32/64) for the width of
        the RWG tiles of the assembly's far-pair kernel,
        "exact_krylov" (0/1) for the FP64-accurate INT8-slice Krylov product,
        "precond_tf32_terms" (3/1) for the TF32 products per complex MAC of the
        complex64 factorisation updates and batched triangular sweeps,
        "gmres_graphs" (0/1) for CUDA-graph replay of GMRES iterations,
        "true_residual" (1 = default: GMRES refines until ||b - Z x|| / ||b||
        meets the tolerance; 0: it stops where Krylov.gmres stops),
        "spin_limit" (polls of a chained triangular-sweep wait before the call
        fails with TimeoutError; negative restores the default),
        "tune_tc_gemm" / "tune_tc_syrk" (0 = autotuned; k pins candidate k:
        256- or 128-wide sweep GEMM tiles or a persistent 256-wide grid;
        4-stage, 2-stage or persistent
        factor-update schedules), "precond_bf16" (1 / 0 / -1 = default: BF16
        instead of TF32 operand pieces for the complex64 factor updates and
        packed sweeps always / never / inside the many-incidence resident
        solves only), "int8_scheme" (0 = default: the FP64-accurate Z X from
        int8 residues modulo 13 coprime moduli, recombined by the Chinese
        remainder theorem; 1: from seven-bit fixed-point slices),
        "tune_int8_tile" (0 = autotuned; 1: one-SM 64 x 256 tiles; 2: CTA-pair
        128 x 256 tiles of the residue-scheme int8 product)."""
        codes = {"tensor_cores": nat.OPT_TENSOR_CORES, "tc_min_rhs": nat.OPT_TC_MIN_RHS,
                 "far_tile": nat.OPT_FAR_TILE, "exact_krylov": nat.OPT_EXACT_KRYLOV,
                 "precond_tf32_terms": nat.OPT_PRECOND_TF32_TERMS, "gmres_graphs": nat.OPT_GMRES_GRAPHS,
                 "true_residual": nat.OPT_TRUE_RESIDUAL, "spin_limit": nat.OPT_SPIN_LIMIT,
                 "tune_tc_gemm": nat.OPT_TUNE_TC_GEMM, "tune_tc_syrk": nat.OPT_TUNE_TC_SYRK,
                 "int8_scheme": nat.OPT_INT8_SCHEME, "tune_int8_tile": nat.OPT_TUNE_INT8_TILE,
                 "precond_bf16": nat.OPT_PRECOND_BF16}
        if name not in codes:
            raise ValueError(f"unknown option {name!r}")
        self.ctx.call("dmb_set_option", codes[name], int(value))
        if name in ("tensor_cores", "precond_tf32_terms", "precond_bf16"):
            self.preconditioner = None

    def far_tile(self) -> int:
        """Far-pair RWG tile width the last assembly used (autotuned unless pinned)."""
        v = ctypes.c_int()
        self.ctx.call("dmb_get_far_tile", ctypes.byref(v))
        return v.value

    # -- impedance matrix -----------------------------------------------
    def assemble(self, k: float, quad_order: int = 3, eta0: float = ETA0_DEFAULT,
                 precision: str = "fp64", copy_out: bool = False):
        if precision not in _PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}")
        Z = np.empty((self.N, self.N), dtype=np.complex128, order="F") if copy_out else None
        self.ctx.call("dmb_assemble_z", float(k), float(eta0), int(quad_order),
                      _PRECISIONS[precision], nat.dptr(Z) if copy_out else None)
        self.k, self.eta0, self.quad_order, self.precision = float(k), float(eta0), quad_order, precision
        self.preconditioner = None
        return Z

    def z_host(self) -> np.ndarray:
        m = np.repeat(np.arange(1, self.N + 1), self.N).astype(np.int64)
        n = np.tile(np.arange(1, self.N + 1), self.N).astype(np.int64)
        return self.entries(m, n).reshape(self.N, self.N)

    def entries(self, m, n) -> np.ndarray:
        m = np.ascontiguousarray(m, dtype=np.int64)
        n = np.ascontiguousarray(n, dtype=np.int64)
        out = np.empty(m.size, dtype=np.complex128)
        self.ctx.call("dmb_z_entries", nat.lptr(m), nat.lptr(n), m.size, nat.dptr(out))
        return out

    def apply_impedance(self, zs_per_triangle) -> None:
        zs = np.ascontiguousarray(np.broadcast_to(np.asarray(zs_per_triangle, dtype=np.complex128),
                                                  (self.mesh.ntriangles,)))
        self.ctx.call("dmb_apply_impedance", nat.dptr(zs))
        self.preconditioner = None

    def matvec(self, x) -> np.ndarray:
        X = nat.c128(x)
        nrhs = 1 if X.ndim == 1 else X.shape[1]
        Y = np.empty_like(X)
        self.ctx.call("dmb_matvec", nat.dptr(X), nat.dptr(Y), nrhs)
        return Y

    # -- preconditioner ---------------------------------------------------
    def build_nearfield(self, cutoff: float, factorization: str = "lu") -> "NearFieldPreconditionerData":
        kinds = {"lu": nat.PRECOND_NF_LU, "diag": nat.PRECOND_NF_DIAG}
        if factorization not in kinds:
            raise ValueError(f"invalid factorization={factorization}; expected one of (:lu, :diag)")
        ratio = ctypes.c_double()
        self.ctx.call("dmb_nf_build", float(cutoff), kinds[factorization], ctypes.byref(ratio))
        self.preconditioner = NearFieldPreconditionerData(self, kinds[factorization], float(cutoff),
                                                          ratio.value)
        return self.preconditioner

    def build_local(self, radius: float, learned: bool = False, mode: str | None = None
                    ) -> "NearFieldPreconditionerData":
        """Sparse right preconditioner from per-RWG near blocks.

        mode "local" (default): exact local-inverse rows; "ring": plus one
        line-searched ring-residual step; "learned" (or learned=True): that
        step with the trained network's per-entry direction; "ls": the
        least-squares sparse-inverse rows the network is trained toward."""
        mode = mode or ("learned" if learned else "local")
        codes = {"local": 0, "learned": 1, "ls": 2, "ring": 3}
        if mode not in codes:
            raise ValueError(f"unknown local preconditioner mode {mode!r}")
        self.ctx.call("dmb_local_build", float(radius), codes[mode])
        kind = {"learned": nat.PRECOND_LEARNED, "ring": nat.PRECOND_RING}.get(mode, nat.PRECOND_LOCAL_INV)
        self.preconditioner = NearFieldPreconditionerData(self, kind, float(radius), 64.0 / self.N)
        return self.preconditioner

    def train_network(self, radius: float, epochs: int = 4, batch: int = 512, lr: float = 2e-3,
                      seed: int = 0) -> float:
        loss = ctypes.c_double()
        self.ctx.call("dmb_net_train", float(radius), int(epochs), int(batch), float(lr), int(seed),
                      ctypes.byref(loss))
        self.preconditioner = None
        return loss.value

    def network_weights(self) -> np.ndarray:
        w = np.empty(self.ctx.lib.dmb_net_param_count(), dtype=np.float32)
        self.ctx.call("dmb_net_get", w.ctypes.data_as(nat._FP))
        return w

    def set_network_weights(self, w) -> None:
        w = np.ascontiguousarray(w, dtype=np.float32)
        if w.size != self.ctx.lib.dmb_net_param_count():
            raise nat.DimensionMismatch("network weight vector has the wrong length")
        self.ctx.call("dmb_net_set", w.ctypes.data_as(nat._FP))

    def save_network(self, path) -> None:
        """Checkpoint: 8-byte magic, int32 count, float32 weights."""
        w = self.network_weights()
        with open(path, "wb") as f:
            f.write(NET_MAGIC)
            f.write(np.int32(w.size).tobytes())
            f.write(w.tobytes())

    def load_network(self, path) -> None:
        with open(path, "rb") as f:
            if f.read(8) != NET_MAGIC:
                raise ValueError("not a diffmom_b200 network checkpoint")
            n = int(np.frombuffer(f.read(4), dtype=np.int32)[0])
            w = np.frombuffer(f.read(4 * n), dtype=np.float32)
        if w.size != n:
            raise ValueError("truncated network checkpoint")
        self.set_network_weights(w)

    def nf_apply(self, x) -> np.ndarray:
        X = nat.c128(x)
        nrhs = 1 if X.ndim == 1 else X.shape[1]
        Y = np.empty_like(X)
        self.ctx.call("dmb_nf_apply", nat.dptr(X), nat.dptr(Y), nrhs)
        return Y

    # -- excitation -------------------------------------------------------
    def plane_wave_rhs(self, kvecs, E0s, pols, quad_order: int = 3) -> np.ndarray:
        kv = np.ascontiguousarray(np.atleast_2d(kvecs), dtype=np.float64)
        pl = np.ascontiguousarray(np.atleast_2d(pols), dtype=np.float64)
        e0 = np.ascontiguousarray(np.atleast_1d(E0s), dtype=np.float64)
        R = kv.shape[0]
        V = np.empty((self.N, R), dtype=np.complex128, order="F")
        self.ctx.call("dmb_rhs_plane_waves", nat.dptr(kv), nat.dptr(e0), nat.dptr(pl), R,
                      int(quad_order), nat.dptr(V))
        return V

    def dipole_rhs(self, positions, moments, types, frequencies, quad_order: int = 3) -> np.ndarray:
        """assemble_dipole (Excitation.jl:2924-2953) for R dipoles at once:
        positions (R, 3), complex moments (R, 3), types 'electric'/'magnetic'
        per dipole, frequencies (R,) in Hz.  Returns V (N, R)."""
        pos = np.ascontiguousarray(np.atleast_2d(positions), dtype=np.float64)
        mom = np.ascontiguousarray(np.atleast_2d(moments), dtype=np.complex128)
        R = pos.shape[0]
        if isinstance(types, str):
            types = [types] * R
        codes = {"electric": 0, "magnetic": 1}
        try:
            mag = np.ascontiguousarray([codes[str(t).lstrip(":")] for t in types], dtype=np.int32)
        except KeyError as e:
            raise ValueError(f"Dipole type must be :electric or :magnetic, got {e.args[0]}") from None
        fr = np.ascontiguousarray(np.broadcast_to(np.asarray(frequencies, dtype=np.float64), (R,)))
        if pos.shape != (R, 3) or mom.shape != (R, 3) or mag.shape != (R,):
            raise ValueError("dipole positions and moments must be (R, 3)")
        V = np.empty((self.N, R), dtype=np.complex128, order="F")
        self.ctx.call("dmb_rhs_dipoles", R, nat.dptr(pos), nat.dptr(mom), nat.iptr(mag), nat.dptr(fr),
                      int(quad_order), nat.dptr(V))
        return V

    def pattern_feed_rhs(self, pattern: "PatternFeedExcitation", quad_order: int = 3) -> np.ndarray:
        """assemble_pattern_feed (Excitation.jl:3044-3071) on the device; V (N,)."""
        th = np.ascontiguousarray(pattern.theta, dtype=np.float64)
        ph = np.ascontiguousarray(pattern.phi, dtype=np.float64)
        ft = np.asfortranarray(pattern.Ftheta, dtype=np.complex128)
        fp = np.asfortranarray(pattern.Fphi, dtype=np.complex128)
        # column-major complex matrices as interleaved doubles
        ftv = np.ascontiguousarray(np.stack([ft.real.ravel(order="F"), ft.imag.ravel(order="F")], 1).ravel())
        fpv = np.ascontiguousarray(np.stack([fp.real.ravel(order="F"), fp.imag.ravel(order="F")], 1).ravel())
        pc = np.ascontiguousarray(pattern.phase_center, dtype=np.float64)
        V = np.empty(self.N, dtype=np.complex128)
        self.ctx.call("dmb_rhs_pattern_feed", th.size, nat.dptr(th), ph.size, nat.dptr(ph), nat.dptr(ftv),
                      nat.dptr(fpv), float(pattern.frequency), nat.dptr(pc),
                      1 if pattern.convention == "exp_minus_iwt" else 0, int(quad_order), nat.dptr(V))
        return V

    def gradient_impedance(self, I, lam, tri_patch, P: int, reactive: bool = False,
                           quad_order: int = 3) -> np.ndarray:
        """gradient_impedance (Adjoint.jl:1081-1119) on the device for 0-based
        per-triangle patch ids; I, lam (N,) or (N, R); returns (P,) or (P, R)."""
        Ia = nat.c128(I)
        La = nat.c128(lam)
        if Ia.shape != La.shape or Ia.shape[0] != self.N:
            raise ValueError(f"I and lambda must both have {self.N} rows and the same shape")
        R = 1 if Ia.ndim == 1 else Ia.shape[1]
        tp = np.ascontiguousarray(tri_patch, dtype=np.int32)
        if tp.shape != (self.mesh.ntriangles,):
            raise ValueError(f"tri_patch length {tp.size} does not match mesh triangle count {self.mesh.ntriangles}")
        g = np.empty((int(P), R), dtype=np.float64, order="F")
        self.ctx.call("dmb_gradient_impedance", R, nat.dptr(Ia), nat.dptr(La), nat.iptr(tp), int(P),
                      1 if reactive else 0, int(quad_order), nat.dptr(g))
        return g[:, 0] if Ia.ndim == 1 else g

    # -- batched resident solve -------------------------------------------
    _PC_CODES = {"none": nat.PRECOND_NONE, "lu": nat.PRECOND_NF_LU, "diag": nat.PRECOND_NF_DIAG,
                 "local": nat.PRECOND_LOCAL_INV, "learned": nat.PRECOND_LEARNED, "ring": nat.PRECOND_RING}

    def solve_many(self, k: float, kvecs, pols, E0s=None, precision: str = "mixed",
                   preconditioner: str = "lu", cutoff: float = math.inf, tol: float = 1e-6,
                   maxiter: int = 300, precond_side: str = "right", quad_order: int = 3,
                   eta0: float = ETA0_DEFAULT, rcs: bool = True):
        """Assemble Z, build the preconditioner, solve all incidences by block
        GMRES and (rcs=True) return the monostatic sigma of each; the currents
        stay on the device (``currents()``)."""
        if precision not in _PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}")
        if preconditioner not in self._PC_CODES:
            raise ValueError(f"unknown preconditioner {preconditioner!r}")
        side = {"left": nat.SIDE_LEFT, "right": nat.SIDE_RIGHT}.get(precond_side)
        if side is None:
            raise ValueError(f"Invalid precond_side: {precond_side} (expected :left or :right)")
        kv = np.ascontiguousarray(np.atleast_2d(kvecs), dtype=np.float64)
        pl = np.ascontiguousarray(np.atleast_2d(pols), dtype=np.float64)
        R = kv.shape[0]
        e0 = np.ascontiguousarray(np.ones(R) if E0s is None else np.broadcast_to(E0s, (R,)), dtype=np.float64)
        if kv.shape != (R, 3) or pl.shape != (R, 3):
            raise nat.DimensionMismatch("kvecs and pols must both be R x 3")
        p = nat.SolveParams()
        p.k, p.eta0, p.cutoff, p.tol = float(k), float(eta0), float(cutoff), float(tol)
        p.quad_order, p.precision, p.precond_kind = int(quad_order), _PRECISIONS[precision], \
            self._PC_CODES[preconditioner]
        p.precond_side, p.maxiter = side, int(maxiter)
        sig = np.empty(R, dtype=np.float64) if rcs else None
        st = nat.GmresStats()
        self.ctx.call("dmb_solve_resident_many", ctypes.byref(p), R, nat.dptr(kv), nat.dptr(e0), nat.dptr(pl),
                      nat.dptr(sig) if rcs else None, ctypes.byref(st))
        self.k, self.eta0, self.quad_order, self.precision = float(k), float(eta0), quad_order, precision
        self._sol_r = R
        return sig, GmresResult(st.niter, bool(st.solved), st.residual, st.true_residual, st.restarts)

    def currents(self) -> np.ndarray:
        """The resident N x R currents of the last solve_many."""
        R = getattr(self, "_sol_r", 0)
        if R < 1:
            raise nat.DiffMoMError("no resident solution")
        I = np.empty((self.N, R), dtype=np.complex128, order="F")
        self.ctx.call("dmb_copy_solution", nat.dptr(I))
        return I

    # -- solvers ----------------------------------------------------------
    def gmres(self, rhs, tol=1e-8, maxiter=200, preconditioner=None, precond_side="left",
              check_gmres_convergence=True, adjoint=False):
        """GMRES on Z x = rhs (adjoint=True: Z^H x = rhs, IterativeSolve.jl:409)."""
        B = nat.c128(rhs)
        nrhs = 1 if B.ndim == 1 else B.shape[1]
        X = np.empty_like(B)
        st = nat.GmresStats()
        kind = nat.PRECOND_NONE if preconditioner is None else preconditioner.kind
        side = {"left": nat.SIDE_LEFT, "right": nat.SIDE_RIGHT}.get(precond_side)
        if side is None:
            raise ValueError(f"Invalid precond_side: {precond_side} (expected :left or :right)")
        fn = self.ctx.lib.dmb_gmres_adjoint if adjoint else self.ctx.lib.dmb_gmres
        status = fn(self.ctx.h, nat.dptr(B), nat.dptr(X), nrhs, float(tol), int(maxiter), kind, side,
                    1 if check_gmres_convergence else 0, ctypes.byref(st))
        self.ctx._check(status)
        return X, GmresResult(st.niter, bool(st.solved), st.residual, st.true_residual, st.restarts)

    def solve_direct(self, rhs):
        B = nat.c128(rhs)
        nrhs = 1 if B.ndim == 1 else B.shape[1]
        X = np.empty_like(B)
        berr = ctypes.c_double()
        self.ctx.call("dmb_solve_direct", nat.dptr(B), nat.dptr(X),
                      nrhs, ctypes.byref(berr))
        self.preconditioner = None
        return X, berr.value

    def farfield(self, rhat, I, k=None, eta0=ETA0_DEFAULT, quad_order=3) -> np.ndarray:
        rh = np.ascontiguousarray(np.atleast_2d(rhat), dtype=np.float64)
        Ic = nat.c128(I)
        nrhs = 1 if Ic.ndim == 1 else Ic.shape[1]
        NO = rh.shape[0]
        E = np.empty((3, NO, nrhs), dtype=np.complex128, order="F")
        kk = self.k if k is None else k
        self.ctx.call("dmb_farfield", nat.dptr(rh), NO, float(kk), float(eta0), int(quad_order),
                      nat.dptr(Ic), nrhs, nat.dptr(E))
        return E[:, :, 0] if nrhs == 1 else E

    def timings(self):
        return self.ctx.timings()

    def close(self):
        self.ctx.close()


@dataclass
class GmresResult:
    niter: int
    solved: bool
    residual: float
    true_residual: float
    restarts: int = 0

    @property
    def residuals(self):
        return [self.residual]


@dataclass
class NearFieldPreconditionerData:
    device: EFIEDevice
    kind: int
    cutoff: float
    nnz_ratio: float


class NearFieldOperator:
    """Callable preconditioner y = Z_nf^-1 x (NearFieldPreconditioner.jl:1034)."""

    def __init__(self, P: NearFieldPreconditionerData):
        self.P = P

    def __matmul__(self, x):
        return self.P.device.nf_apply(x)

    def apply(self, x):
        return self.P.device.nf_apply(x)


class NearFieldAdjointOperator:
    """y = (Z_nf^-1)^H x (NearFieldPreconditioner.jl:1237-1290); Z_nf is complex
    symmetric, so this is conj(Z_nf^-1 conj(x))."""

    def __init__(self, P: NearFieldPreconditionerData):
        self.P = P

    def __matmul__(self, x):
        return self.apply(x)

    def apply(self, x):
        return np.conj(self.P.device.nf_apply(np.conj(nat.c128(x))))


# ---------------------------------------------------------------------------
# Julia-named entry points
# ---------------------------------------------------------------------------
def assemble_Z_efie(mesh: TriMesh, rwg: RWGData, k, quad_order: int = 3, eta0=ETA0_DEFAULT,
                    precision: str = "fp64", device: EFIEDevice | None = None) -> np.ndarray:
    """Dense EFIE matrix Z (N x N complex128); EFIE.jl:699-753."""
    dev = device or EFIEDevice(mesh, rwg)
    try:
        return dev.assemble(k, quad_order=quad_order, eta0=eta0, precision=precision, copy_out=True)
    finally:
        if device is None:
            dev.close()


class MatrixFreeEFIEOperator:
    """y = Z x with entries recomputed on the device per product (EFIE.jl:759-909)."""

    def __init__(self, mesh, rwg, k, quad_order=3, eta0=ETA0_DEFAULT):
        self.dev = EFIEDevice(mesh, rwg)
        self.dev.ctx.call("dmb_prepare_operator", float(k), float(eta0), int(quad_order))
        self.shape = (rwg.nedges, rwg.nedges)

    def __matmul__(self, x):
        xc = np.ascontiguousarray(np.asarray(x, dtype=np.complex128))
        y = np.empty_like(xc)
        self.dev.ctx.call("dmb_matvec_free", nat.dptr(xc), nat.dptr(y))
        return y

    def mul(self, x):
        return self @ x


def matrixfree_efie_operator(mesh, rwg, k, quad_order=3, eta0=ETA0_DEFAULT):
    return MatrixFreeEFIEOperator(mesh, rwg, k, quad_order=quad_order, eta0=eta0)


@dataclass
class PlaneWaveExcitation:
    k_vec: np.ndarray
    E0: float
    pol: np.ndarray


def make_plane_wave(k_vec, E0, pol) -> PlaneWaveExcitation:
    """Excitation.jl:97-101 with the validation of Excitation.jl:1549-1616."""
    kv = np.asarray(k_vec, dtype=np.float64).reshape(3)
    pl = np.asarray(pol, dtype=np.float64).reshape(3)
    if not np.all(np.isfinite(kv)):
        raise ValueError("plane-wave k_vec components must be finite.")
    if not math.isfinite(float(E0)):
        raise ValueError(f"plane-wave amplitude E0 must be finite, got {E0}.")
    kn = float(np.linalg.norm(kv))
    if not kn > 0:
        raise ValueError("plane-wave k_vec must have a finite, nonzero norm.")
    pn = float(np.linalg.norm(pl))
    if not math.isclose(pn, 1.0, rel_tol=1e-10, abs_tol=1e-12):
        raise ValueError(f"plane-wave polarization must be a unit vector; norm={pn}.")
    if abs(float(kv @ pl)) / (kn * pn) > 1e-10:
        raise ValueError("plane-wave polarization must be transverse to k_vec")
    return PlaneWaveExcitation(kv, float(E0), pl)


def assemble_plane_wave(mesh, rwg, pw: PlaneWaveExcitation, quad_order=3, device=None) -> np.ndarray:
    dev = device or EFIEDevice(mesh, rwg)
    try:
        return dev.plane_wave_rhs(pw.k_vec[None], [pw.E0], pw.pol[None], quad_order)[:, 0]
    finally:
        if device is None:
            dev.close()


@dataclass
class DipoleExcitation:
    """Excitation.jl:130-136: electric (C m) or magnetic (A m^2) dipole."""
    position: np.ndarray
    moment: np.ndarray
    orientation: np.ndarray
    type: str
    frequency: float


@dataclass
class LoopExcitation:
    """Excitation.jl:143-149: small circular loop of current I, radiating as
    the magnetic dipole I pi a^2 n."""
    center: np.ndarray
    normal: np.ndarray
    radius: float
    current: complex
    frequency: float

    def equivalent_moment(self) -> np.ndarray:
        """_loop_equivalent_moment (Excitation.jl:936-942)."""
        return complex(self.current) * math.pi * self.radius ** 2 * self.normal.astype(np.complex128)


def _finite_vec3(v, what, dtype=np.float64):
    a = np.asarray(v, dtype=dtype).reshape(3)
    if not np.all(np.isfinite(a)):
        raise ValueError(f"{what} must have finite components.")
    return a


def _unit_vec3(v, what):
    a = _finite_vec3(v, what)
    n = float(np.linalg.norm(a))
    if not (math.isfinite(n) and math.isclose(n, 1.0, rel_tol=1e-10, abs_tol=1e-12)):
        raise ValueError(f"{what} must be a unit vector; norm={n}.")
    return a


def _positive_frequency(f, what):
    f = float(f)
    if not (math.isfinite(f) and f > 0.0):
        raise ValueError(f"{what} frequency must be finite and positive, got {f}.")
    return f


def make_dipole(position, moment, orientation, type, frequency=1e9) -> DipoleExcitation:
    """Excitation.jl:313-317 with the validation of Excitation.jl:1662-1678."""
    pos = _finite_vec3(position, "DipoleExcitation position")
    mom = _finite_vec3(moment, "DipoleExcitation moment", np.complex128)
    ori = _unit_vec3(orientation, "DipoleExcitation orientation")
    t = str(type).lstrip(":")
    if t not in ("electric", "magnetic"):
        raise ValueError(f"DipoleExcitation type must be :electric or :magnetic, got {type}.")
    return DipoleExcitation(pos, mom, ori, t, _positive_frequency(frequency, "DipoleExcitation"))


def make_loop(center, normal, radius, current, frequency=1e9) -> LoopExcitation:
    """Excitation.jl:319-323 with the validation of Excitation.jl:1680-1698."""
    c = _finite_vec3(center, "LoopExcitation center")
    n = _unit_vec3(normal, "LoopExcitation normal")
    a = float(radius)
    if not (math.isfinite(a) and a > 0.0):
        raise ValueError(f"LoopExcitation radius must be finite and positive, got {radius}.")
    cur = complex(current)
    if not (math.isfinite(cur.real) and math.isfinite(cur.imag)):
        raise ValueError(f"LoopExcitation current must be finite, got {current}.")
    return LoopExcitation(c, n, a, cur, _positive_frequency(frequency, "LoopExcitation"))


def _as_dipole(e):
    if isinstance(e, LoopExcitation):
        return e.center, e.equivalent_moment(), "magnetic", e.frequency
    return e.position, e.moment, e.type, e.frequency


def _with_device(mesh, rwg, device, fn):
    dev = device or EFIEDevice(mesh, rwg)
    try:
        return fn(dev)
    finally:
        if device is None:
            dev.close()


def assemble_dipole(mesh, rwg, dipole: DipoleExcitation, quad_order=3, device=None) -> np.ndarray:
    """Excitation.jl:2924-2953 on the device."""
    p, m, t, f = _as_dipole(dipole)
    return _with_device(mesh, rwg, device, lambda d: d.dipole_rhs(p[None], m[None], [t], [f], quad_order)[:, 0])


def assemble_loop(mesh, rwg, loop: LoopExcitation, quad_order=3, device=None) -> np.ndarray:
    """Excitation.jl:2955-2977: the loop's equivalent magnetic dipole."""
    return assemble_dipole(mesh, rwg, loop, quad_order=quad_order, device=device)


@dataclass
class PatternFeedExcitation:
    """Excitation.jl:262-280: field synthesised from far-field coefficients on a
    spherical grid, E(r) = exp(-ikR)/R (F_theta e_theta + F_phi e_phi) about
    phase_center; theta/phi in radians, F of shape (len(theta), len(phi))."""
    theta: np.ndarray
    phi: np.ndarray
    Ftheta: np.ndarray
    Fphi: np.ndarray
    frequency: float
    phase_center: np.ndarray
    convention: str


_PATTERN_CONVENTIONS = ("exp_plus_iwt", "exp_minus_iwt")


def _validate_pattern_grid(theta, phi):
    """_validate_pattern_grid (Excitation.jl:999-1025)."""
    if theta.size < 2:
        raise ValueError("Pattern feed requires at least 2 theta samples.")
    if phi.size < 2:
        raise ValueError("Pattern feed requires at least 2 phi samples.")
    if not np.all(np.isfinite(theta)):
        raise ValueError("Theta grid contains non-finite values.")
    if not np.all(np.isfinite(phi)):
        raise ValueError("Phi grid contains non-finite values.")
    if not np.all(np.diff(theta) > 0):
        raise ValueError("Theta grid must be strictly increasing.")
    if not np.all(np.diff(phi) > 0):
        raise ValueError("Phi grid must be strictly increasing.")
    if theta[0] < -1e-12 or theta[-1] > math.pi + 1e-12:
        raise ValueError(f"Theta grid must lie in [0, pi] (radians). Got range [{theta[0]}, {theta[-1]}].")
    span = phi[-1] - phi[0]
    if span <= 0:
        raise ValueError("Phi grid span must be positive.")
    if span >= 2 * math.pi - 1e-12:
        raise ValueError("Phi grid should cover one open 2 pi period without a duplicate endpoint "
                         "(e.g., 0:d:2 pi - d).")


def _pattern_metadata(frequency, phase_center, convention):
    """_validated_pattern_feed_metadata (Excitation.jl:1067-1081)."""
    f = float(frequency)
    if not (math.isfinite(f) and f > 0.0):
        raise ValueError(f"Pattern feed frequency must be finite and positive, got {frequency}.")
    pc = np.asarray(phase_center, dtype=np.float64).reshape(3)
    if not np.all(np.isfinite(pc)):
        raise ValueError("Pattern feed phase_center must be finite.")
    conv = str(convention).lstrip(":")
    if conv not in _PATTERN_CONVENTIONS:
        raise ValueError(f"Unsupported pattern convention: {convention} (expected :exp_plus_iwt or :exp_minus_iwt).")
    return f, pc, conv


def make_pattern_feed(theta, phi, Ftheta, Fphi, frequency, phase_center=(0.0, 0.0, 0.0),
                      angles_in_degrees=False, convention="exp_plus_iwt") -> PatternFeedExcitation:
    """Excitation.jl:1084-1128."""
    f, pc, conv = _pattern_metadata(frequency, phase_center, convention)
    th = np.array(theta, dtype=np.float64)
    ph = np.array(phi, dtype=np.float64)
    if angles_in_degrees:
        th *= math.pi / 180
        ph *= math.pi / 180
    _validate_pattern_grid(th, ph)
    ft = np.asarray(Ftheta, dtype=np.complex128)
    fp = np.asarray(Fphi, dtype=np.complex128)
    for name, m in (("Ftheta", ft), ("Fphi", fp)):
        if m.shape != (th.size, ph.size):
            raise ValueError(f"{name} has shape {m.shape}, expected {(th.size, ph.size)}.")
        if not np.all(np.isfinite(m)):
            raise ValueError(f"{name} contains non-finite coefficients.")
    return PatternFeedExcitation(th, ph, ft.copy(), fp.copy(), f, pc, conv)


_EPS0 = 8.854187817e-12
_ETA0 = math.sqrt(4 * math.pi * 1e-7 / _EPS0)
_C0_PATTERN = 299792458.0


def _spherical_basis(theta, phi):
    st, ct, sp, cp = np.sin(theta), np.cos(theta), np.sin(phi), np.cos(phi)
    rhat = np.stack([st * cp, st * sp, ct], -1)
    et = np.stack([ct * cp, ct * sp, -st], -1)
    ep = np.stack([-sp, cp, np.zeros_like(sp)], -1)
    return rhat, et, ep


def make_analytic_dipole_pattern_feed(dipole: DipoleExcitation, theta, phi, phase_center=None,
                                      angles_in_degrees=False, convention="exp_plus_iwt") -> PatternFeedExcitation:
    """Excitation.jl:1468-1509: the dipole's far-field coefficients
    (_dipole_farfield_unphased, :898-...) sampled on the grid; electric:
    k^2 / (4 pi eps0) (rhat x p) x rhat, magnetic: eta0 k^2 / (4 pi) (m x rhat)."""
    pc = dipole.position if phase_center is None else phase_center
    f, pc, conv = _pattern_metadata(dipole.frequency, pc, convention)
    k = 2 * math.pi * f / _C0_PATTERN
    th = np.array(theta, dtype=np.float64)
    ph = np.array(phi, dtype=np.float64)
    if angles_in_degrees:
        th *= math.pi / 180
        ph *= math.pi / 180
    _validate_pattern_grid(th, ph)
    T, P = np.meshgrid(th, ph, indexing="ij")
    rhat, et, ep = _spherical_basis(T, P)
    p = np.asarray(dipole.moment, dtype=np.complex128)
    if dipole.type == "electric":
        F = np.cross(np.cross(rhat, p), rhat) * (k * k / (4 * math.pi * _EPS0))
    else:
        F = np.cross(p, rhat) * (_ETA0 * k * k / (4 * math.pi))
    Ft = np.sum(F * et, -1)
    Fp = np.sum(F * ep, -1)
    return PatternFeedExcitation(th, ph, Ft, Fp, f, pc, conv)


def assemble_pattern_feed(mesh, rwg, pattern: PatternFeedExcitation, quad_order=3, device=None) -> np.ndarray:
    """Excitation.jl:3044-3071 on the device."""
    return _with_device(mesh, rwg, device, lambda d: d.pattern_feed_rhs(pattern, quad_order))


_EXCITATION_TYPES = (PlaneWaveExcitation, DipoleExcitation, LoopExcitation, PatternFeedExcitation)


def assemble_excitation(mesh, rwg, excitation, quad_order=3, device=None) -> np.ndarray:
    if not isinstance(excitation, _EXCITATION_TYPES):
        raise TypeError(f"Unsupported excitation type: {type(excitation).__name__}")
    return assemble_multiple_excitations(mesh, rwg, [excitation], quad_order=quad_order, device=device)[:, 0]


def assemble_multiple_excitations(mesh, rwg, excitations, quad_order=3, device=None) -> np.ndarray:
    """One column per excitation; plane waves and dipoles/loops are each
    assembled in one launch, pattern feeds one launch each."""
    excitations = list(excitations)
    for e in excitations:
        if not isinstance(e, _EXCITATION_TYPES):
            raise TypeError(f"Unsupported excitation type: {type(e).__name__}")

    def run(dev):
        V = np.empty((dev.N, len(excitations)), dtype=np.complex128, order="F")
        pw = [i for i, e in enumerate(excitations) if isinstance(e, PlaneWaveExcitation)]
        dp = [i for i, e in enumerate(excitations) if isinstance(e, (DipoleExcitation, LoopExcitation))]
        for i, e in enumerate(excitations):
            if isinstance(e, PatternFeedExcitation):
                V[:, i] = dev.pattern_feed_rhs(e, quad_order)
        if pw:
            es = [excitations[i] for i in pw]
            V[:, pw] = dev.plane_wave_rhs(np.stack([e.k_vec for e in es]), np.array([e.E0 for e in es]),
                                          np.stack([e.pol for e in es]), quad_order)
        if dp:
            src = [_as_dipole(excitations[i]) for i in dp]
            V[:, dp] = dev.dipole_rhs(np.stack([s[0] for s in src]), np.stack([s[1] for s in src]),
                                      [s[2] for s in src], np.array([s[3] for s in src]), quad_order)
        return V

    return _with_device(mesh, rwg, device, run)


# ---------------------------------------------------------------------------
# solvers
# ---------------------------------------------------------------------------
def build_nearfield_preconditioner(device, cutoff: float | None = None, factorization: str = "lu",
                                   precision: str = "fp64"):
    """NearFieldPreconditioner.jl:670-758 for a device with an assembled Z and
    a distance cutoff; for an ACAOperator (NearFieldPreconditioner.jl:952-1000)
    the near field is the operator's dense blocks and `cutoff` is unused."""
    from .aca import ACAOperator
    if isinstance(device, ACAOperator):
        return device.build_nearfield(factorization, precision)
    if cutoff is None:
        raise ValueError("build_nearfield_preconditioner: a cutoff is required for a dense operator")
    return device.build_nearfield(cutoff, factorization)


def solve_gmres(device, rhs, preconditioner=None, precond_side="left", tol=1e-8,
                maxiter=200, check_gmres_convergence=True):
    """IterativeSolve.jl: GMRES on the dense Z of an EFIEDevice or on an
    ACAOperator's H-matrix."""
    return device.gmres(rhs, tol=tol, maxiter=maxiter, preconditioner=preconditioner,
                        precond_side=precond_side, check_gmres_convergence=check_gmres_convergence)


def solve_gmres_adjoint(device, rhs, preconditioner=None, precond_side="left", tol=1e-8,
                        maxiter=200, check_gmres_convergence=True):
    """IterativeSolve.jl:409-470: GMRES on Z^H x = rhs with the adjoint
    near-field preconditioner (dense Z or an ACAOperator)."""
    return device.gmres(rhs, tol=tol, maxiter=maxiter, preconditioner=preconditioner,
                        precond_side=precond_side, check_gmres_convergence=check_gmres_convergence, adjoint=True)


def solve_adjoint_rhs(device: EFIEDevice, rhs, preconditioner=None, gmres_precond_side="left", gmres_tol=1e-8,
                      gmres_maxiter=200, check_gmres_convergence=True, check_true_residual=True,
                      true_residual_factor=100.0):
    """Adjoint.jl:1029-1078 (solver=:gmres): Z^H lambda = rhs on the device;
    with check_true_residual the FP64 residual must stay within
    true_residual_factor x gmres_tol."""
    lam, stats = solve_gmres_adjoint(device, rhs, preconditioner=preconditioner, precond_side=gmres_precond_side,
                                     tol=gmres_tol, maxiter=gmres_maxiter,
                                     check_gmres_convergence=check_gmres_convergence)
    if check_true_residual and not (stats.true_residual <= true_residual_factor * gmres_tol):
        raise nat.NotConvergedError(f"adjoint true residual {stats.true_residual:.3e} exceeds "
                                f"{true_residual_factor} x tol {gmres_tol:.1e}")
    return lam


@dataclass
class PatchPartition:
    """Types.jl:1263-1280: tri_patch[t] in 1..P is the patch of triangle t."""
    tri_patch: np.ndarray
    P: int

    def __post_init__(self):
        self.tri_patch = np.asarray(self.tri_patch, dtype=np.int64)
        if self.P < 0:
            raise ValueError(f"partition.P must be nonnegative, got {self.P}")
        if self.tri_patch.size and (self.tri_patch.min() < 1 or self.tri_patch.max() > self.P):
            raise ValueError(f"partition.tri_patch entries must lie in 1:{self.P}")


@dataclass
class PatchMass:
    """The patch mass matrices of precompute_patch_mass (Impedance.jl:304-377)
    held implicitly: their entries are evaluated per triangle on the device
    whenever a gradient needs them."""
    device: EFIEDevice
    partition: PatchPartition
    quad_order: int

    def __len__(self):
        return self.partition.P


def precompute_patch_mass(mesh, rwg, partition: PatchPartition, quad_order=3, device=None) -> PatchMass:
    """Impedance.jl:304-377.  The returned object refers to `device` (a new
    EFIEDevice for mesh / rwg when None)."""
    if partition.tri_patch.size != mesh.ntriangles:
        raise ValueError(f"partition.tri_patch length {partition.tri_patch.size} does not match mesh triangle "
                         f"count {mesh.ntriangles}")
    return PatchMass(device or EFIEDevice(mesh, rwg), partition, int(quad_order))


def gradient_impedance(Mp: PatchMass, I, lam, reactive=False) -> np.ndarray:
    """Adjoint.jl:1081-1119: g[p] = 2 Re(lambda^H M_p I) (resistive,
    Z_s = theta_p) or -2 Im(lambda^H M_p I) (reactive, Z_s = i theta_p)."""
    for name, v in (("I", I), ("lambda", lam)):
        if not np.all(np.isfinite(np.asarray(v))):
            raise ValueError(f"{name} must contain only finite values")
    return Mp.device.gradient_impedance(I, lam, Mp.partition.tri_patch - 1, Mp.partition.P, reactive,
                                        Mp.quad_order)


def solve_forward(device: EFIEDevice, v, solver="direct"):
    if solver != "direct":
        raise ValueError("solve_forward: only solver=:direct is provided on the device")
    x, _ = device.solve_direct(v)
    return x


@dataclass
class ScatteringResult:
    I_coeffs: np.ndarray
    method: str
    N: int
    assembly_time_s: float
    solve_time_s: float
    preconditioner_time_s: float
    gmres_iters: int
    gmres_residual: float
    true_residual: float = float("nan")
    warnings: list = field(default_factory=list)
    timings: dict = field(default_factory=dict)


def tune_report() -> str:
    """The online autotuner's measurements and choices so far (this process)."""
    lib = nat.load_library()
    n = ctypes.c_size_t()
    nat.check_free(lib, lib.dmb_tune_report(None, 0, ctypes.byref(n)))
    buf = ctypes.create_string_buffer(n.value + 1)
    nat.check_free(lib, lib.dmb_tune_report(buf, n.value + 1, ctypes.byref(n)))
    return buf.value.decode()


def solve_scattering(mesh: TriMesh, freq_hz, excitation, method: str = "auto",
                     dense_direct_limit: int = 2000, dense_gmres_limit: int = 10000,
                     mlfma_threshold: int = 50000, max_dense_matrix_bytes: int = 2_000_000_000,
                     gmres_tol: float = 1e-6, gmres_maxiter: int = 300,
                     check_gmres_convergence: bool = True, nf_cutoff_lambda: float = 1.0,
                     preconditioner: str = "auto", precond_side: str = "left", quad_order: int = 3,
                     c0: float = C0_DEFAULT, precision: str = "fp64", surface_impedance=None,
                     verbose: bool = False, device: EFIEDevice | None = None, rwg: RWGData | None = None,
                     aca_tol: float = 1e-6, aca_leaf_size: int = 64, aca_eta: float = 1.5,
                     aca_max_rank: int = 50, local_radius_lambda: float = 0.2, network=None):
    """Workflow.jl:67-317 on the GPU.

    method: "auto" | "dense_direct" | "dense_gmres" | "aca_gmres".  "auto"
    selects as the reference does (Workflow.jl:147-160): dense_direct up to
    dense_direct_limit unknowns, dense_gmres up to dense_gmres_limit,
    aca_gmres up to mlfma_threshold; above it the reference's MLFMA, which
    this library does not provide (ValueError).  On a B200 the dense methods
    are faster than the H-matrix at every size the reference sends to ACA
    (N <= 50,000 fits in HBM): pass method="dense_gmres" (or a larger
    dense_gmres_limit) to keep them.  The dense methods check the matrix
    payload (N^2 x 16 bytes in FP64, x 8 in mixed precision) against
    max_dense_matrix_bytes before assembly, as the reference does
    (Workflow.jl:169-174).  "aca_gmres" runs the reference's H-matrix path
    (build_aca_operator with the aca_* parameters, near-field preconditioner
    from its dense blocks).  precision "fp64" is the plain path; "mixed"
    assembles far pairs in FP32 (complex64 Z) and factors the preconditioner
    in FP32 while GMRES keeps FP64 Arnoldi and residuals (for aca_gmres only
    the preconditioner is complex64).  GMRES tests convergence on the
    unpreconditioned FP64 residual (refining a left-preconditioned solve until
    it passes).

    preconditioner: "auto" / "lu" / "diag" / "none" as the reference
    (near-field LU at nf_cutoff_lambda wavelengths), plus two sparse right
    preconditioners of this library for the dense GMRES path, built from each
    RWG's near block within local_radius_lambda wavelengths (<= 64
    neighbours): "local" (exact local-inverse rows) and "learned" (those rows
    corrected by one ring-residual step whose direction the trained network
    modulates; weights from ``network`` -- a checkpoint path or a weight
    vector -- else the library's default weights, diffmom_b200/learned.py).
    Both are applied on the right whatever precond_side says.  If GMRES with
    either does not reach gmres_tol within gmres_maxiter, the near-field LU
    preconditioner is built and the system solved again with it (the
    fallback; a warning says so).
    """
    f = float(freq_hz)
    if not (math.isfinite(f) and f > 0):
        raise ValueError(f"solve_scattering: freq_hz must be finite and positive, got {freq_hz}")
    if method not in ("auto", "dense_direct", "dense_gmres", "aca_gmres"):
        raise ValueError("solve_scattering: method must be :auto, :dense_direct, :dense_gmres, or :aca_gmres "
                         "(:mlfma is not provided by this library)")
    if dense_direct_limit < 0:
        raise ValueError(f"solve_scattering: dense_direct_limit must be nonnegative, got {dense_direct_limit}")
    if dense_gmres_limit < dense_direct_limit:
        raise ValueError(f"solve_scattering: dense_gmres_limit ({dense_gmres_limit}) must be at least "
                         f"dense_direct_limit ({dense_direct_limit})")
    if mlfma_threshold < dense_gmres_limit:
        raise ValueError(f"solve_scattering: mlfma_threshold ({mlfma_threshold}) must be at least "
                         f"dense_gmres_limit ({dense_gmres_limit})")
    if not (isinstance(max_dense_matrix_bytes, (int, np.integer)) and max_dense_matrix_bytes > 0):
        raise ValueError(f"max_dense_matrix_bytes must be a positive integer, got {max_dense_matrix_bytes}")
    if preconditioner not in ("auto", "lu", "diag", "none", "local", "learned"):
        raise ValueError("solve_scattering: preconditioner must be :auto, :lu, :diag, :none, :local or :learned")
    if not (math.isfinite(local_radius_lambda) and local_radius_lambda > 0):
        raise ValueError(f"solve_scattering: local_radius_lambda must be finite and positive, got "
                         f"{local_radius_lambda}")
    if method == "aca_gmres" and surface_impedance is not None:
        raise ValueError("solve_scattering: surface_impedance is not supported by :aca_gmres")
    lam = c0 / f
    k = _frequency_to_wavenumber(f, c0)
    warnings = []
    if isinstance(excitation, PlaneWaveExcitation):
        kn = float(np.linalg.norm(excitation.k_vec))
        if abs(kn - k) > 1e-8 * k:
            raise ValueError("solve_scattering: plane-wave |k_vec| must equal 2*pi*freq/c0")
    if mesh_edge_max(mesh) / lam > 0.1:
        warnings.append("Mesh under-resolved")
    rwg = rwg if rwg is not None else build_rwg(mesh)
    N = rwg.nedges
    if N < 1:
        raise ValueError("solve_scattering: mesh produces no RWG unknowns")
    sel = method
    if method == "auto":
        if N <= dense_direct_limit:
            sel = "dense_direct"
        elif N <= dense_gmres_limit:
            sel = "dense_gmres"
        elif N <= mlfma_threshold:
            sel = "aca_gmres"
        else:
            raise ValueError(f"solve_scattering: N={N} is above mlfma_threshold={mlfma_threshold}; the MLFMA "
                             "path is not provided by this library (pass method=\"aca_gmres\" or "
                             "\"dense_gmres\")")
        if sel == "aca_gmres" and surface_impedance is not None:
            raise ValueError("solve_scattering: surface_impedance is not supported by :aca_gmres "
                             "(auto-selected above dense_gmres_limit; pass method=\"dense_gmres\")")
    if preconditioner in ("local", "learned") and sel != "dense_gmres":
        raise ValueError(f"solve_scattering: preconditioner :{preconditioner} needs method :dense_gmres "
                         f"(selected :{sel})")
    if sel in ("dense_direct", "dense_gmres"):
        payload = N * N * (16 if precision == "fp64" else 8)
        if payload > max_dense_matrix_bytes:
            raise ValueError(f"solve_scattering dense EFIE matrix requires {payload} raw bytes, exceeding "
                             f"max_dense_matrix_bytes={max_dense_matrix_bytes}")
    dev = device or EFIEDevice(mesh, rwg)
    own = device is None
    try:
        if isinstance(excitation, PlaneWaveExcitation):
            v = dev.plane_wave_rhs(excitation.k_vec[None], [excitation.E0], excitation.pol[None],
                                   quad_order)[:, 0]
        else:
            v = np.asarray(excitation, dtype=np.complex128)
            if v.shape != (N,):
                raise nat.DimensionMismatch(f"solve_scattering: excitation length {v.size} != N={N}")
        t0 = time.perf_counter()
        aca_op = None
        if sel == "aca_gmres":
            from .aca import build_aca_operator
            aca_op = build_aca_operator(mesh, rwg, k, leaf_size=aca_leaf_size, eta=aca_eta, aca_tol=aca_tol,
                                        max_rank=aca_max_rank, quad_order=quad_order, device=dev)
        else:
            dev.assemble(k, quad_order=quad_order, precision=precision)
            if surface_impedance is not None:
                dev.apply_impedance(surface_impedance)
        t_asm = time.perf_counter() - t0
        t_pc = 0.0
        iters, resid, tres = -1, float("nan"), float("nan")
        t1 = time.perf_counter()
        if aca_op is not None:
            pc_used = "lu" if preconditioner == "auto" else preconditioner
            P = None
            if pc_used != "none":
                tp = time.perf_counter()
                P = aca_op.build_nearfield(pc_used, precision)
                t_pc = time.perf_counter() - tp
            t1 = time.perf_counter()
            I, st = aca_op.gmres(v, tol=gmres_tol, maxiter=gmres_maxiter, preconditioner=P,
                                 precond_side=precond_side, check_gmres_convergence=check_gmres_convergence)
            iters, resid, tres = st.niter, st.residual, st.true_residual
        elif sel == "dense_direct":
            I, berr = dev.solve_direct(v)
            tres = berr
        else:
            pc_used = "lu" if preconditioner == "auto" else preconditioner
            P = None
            side = precond_side
            if pc_used in ("local", "learned"):
                tp = time.perf_counter()
                if pc_used == "learned":
                    if network is None:
                        from .learned import load_default_network
                        load_default_network(dev)
                    elif isinstance(network, (str, bytes)) or hasattr(network, "__fspath__"):
                        dev.load_network(network)
                    else:
                        dev.set_network_weights(network)
                P = dev.build_local(local_radius_lambda * lam, mode=pc_used)
                t_pc = time.perf_counter() - tp
                side = "right"
            elif pc_used != "none":
                tp = time.perf_counter()
                P = dev.build_nearfield(nf_cutoff_lambda * lam, pc_used)
                t_pc = time.perf_counter() - tp
            t1 = time.perf_counter()
            local = pc_used in ("local", "learned")
            I, st = dev.gmres(v, tol=gmres_tol, maxiter=gmres_maxiter, preconditioner=P,
                              precond_side=side, check_gmres_convergence=check_gmres_convergence and not local)
            if local and not st.solved:
                # the near-field sparse preconditioner is the fallback
                warnings.append(f"GMRES with the {pc_used} preconditioner did not converge in {st.niter} "
                                f"iterations; solved again with the near-field LU preconditioner")
                tp = time.perf_counter()
                P = dev.build_nearfield(nf_cutoff_lambda * lam, "lu")
                t_pc += time.perf_counter() - tp
                I, st2 = dev.gmres(v, tol=gmres_tol, maxiter=gmres_maxiter, preconditioner=P,
                                   precond_side=precond_side, check_gmres_convergence=False)
                st = GmresResult(st.niter + st2.niter, st2.solved, st2.residual, st2.true_residual,
                                 st.restarts + st2.restarts)
                if check_gmres_convergence and not st.solved:
                    raise nat.NotConvergedError(
                        f"GMRES did not converge: niter={st.niter}, true residual {st.true_residual:.3e}, "
                        f"tol={gmres_tol} (the {pc_used} preconditioner and its near-field LU fallback)")
            iters, resid, tres = st.niter, st.residual, st.true_residual
        t_solve = time.perf_counter() - t1
        tm = dev.timings()
        return ScatteringResult(I_coeffs=np.asarray(I).reshape(N), method=sel, N=N,
                                assembly_time_s=t_asm, solve_time_s=t_solve,
                                preconditioner_time_s=t_pc, gmres_iters=iters,
                                gmres_residual=resid, true_residual=tres, warnings=warnings,
                                timings={f: getattr(tm, f) for f, _ in nat.Timings._fields_})
    finally:
        if own:
            dev.close()


@dataclass
class MonostaticResult:
    sigma: np.ndarray            # (R,) monostatic RCS, m^2
    gmres_iters: int
    true_residual: float         # max over incidences of ||b - Z x|| / ||b||
    refinements: int
    currents: np.ndarray | None  # N x R when requested


def monostatic_rcs_sweep(mesh: TriMesh, freq_hz, excitations, precision: str = "mixed",
                         preconditioner: str = "lu", nf_cutoff_lambda: float = math.inf,
                         gmres_tol: float = 1e-6, gmres_maxiter: int = 300, precond_side: str = "right",
                         quad_order: int = 3, c0: float = C0_DEFAULT, return_currents: bool = False,
                         device: EFIEDevice | None = None, rwg: RWGData | None = None) -> MonostaticResult:
    """Monostatic RCS over many plane-wave incidences: what a loop of
    solve_scattering (Workflow.jl:67-317) + backscatter_rcs (Diagnostics.jl:
    476-517) per incidence computes, with Z and its preconditioner built once
    and all incidences solved together by block GMRES on the device.

    With nf_cutoff_lambda = inf the preconditioner is the complete complex64
    LDL^T of Z (GMRES with FP64-residual refinement); a finite cutoff gives
    the reference's near-field preconditioner."""
    f = float(freq_hz)
    if not (math.isfinite(f) and f > 0):
        raise ValueError(f"monostatic_rcs_sweep: freq_hz must be finite and positive, got {freq_hz}")
    k = _frequency_to_wavenumber(f, c0)
    exc = list(excitations)
    if not exc or not all(isinstance(e, PlaneWaveExcitation) for e in exc):
        raise ValueError("monostatic_rcs_sweep: excitations must be a non-empty list of plane waves")
    kvecs = np.array([e.k_vec for e in exc], dtype=np.float64)
    pols = np.array([e.pol for e in exc], dtype=np.float64)
    e0s = np.array([e.E0 for e in exc], dtype=np.float64)
    if np.any(np.abs(np.linalg.norm(kvecs, axis=1) - k) > 1e-8 * k):
        raise ValueError("monostatic_rcs_sweep: plane-wave |k_vec| must equal 2*pi*freq/c0")
    rwg = rwg if rwg is not None else build_rwg(mesh)
    dev = device or EFIEDevice(mesh, rwg)
    own = device is None
    try:
        lam = c0 / f
        sig, st = dev.solve_many(k, kvecs, pols, e0s,
                                 precision=precision, preconditioner=preconditioner,
                                 cutoff=nf_cutoff_lambda * lam, tol=gmres_tol, maxiter=gmres_maxiter,
                                 precond_side=precond_side, quad_order=quad_order)
        cur = dev.currents() if return_currents else None
        return MonostaticResult(sig, st.niter, st.true_residual, st.restarts, cur)
    finally:
        if own:
            dev.close()


@dataclass
class BatchSurface:
    mesh: TriMesh
    rwg: RWGData
    excitation: "PlaneWaveExcitation"
    zs: np.ndarray | None = None   # per-triangle complex surface impedance (ohm), None = PEC


@dataclass
class BatchResult:
    sigma: np.ndarray          # monostatic RCS per surface, m^2
    gmres_iters: np.ndarray
    true_residual: np.ndarray
    latency_ms: np.ndarray     # device time from the batch start to each surface's end
    solve_ms: np.ndarray       # device time of each surface's stages after the batch-wide assembly
    device_ms: float           # device time of the whole batch
    N: np.ndarray
    currents: list | None
    assembly_ms: float = 0.0   # device time of the batch-wide assembly (one far-pair launch for all surfaces)


class SurfaceBatch:
    """Many independent surfaces (each its own mesh, basis, impedance and
    plane wave): every surface's impedance matrix assembled by one far-pair
    launch (plus one launch each for the near terms), then the per-surface
    stages on `lanes` concurrent host threads and streams, largest first."""

    def __init__(self, lanes: int = 8, device: int = 0):
        self.lib = nat.load_library()
        h = ctypes.c_void_p()
        st = self.lib.dmb_batch_create(int(device), int(lanes), ctypes.byref(h))
        if st != nat.DMB_OK:
            raise nat.DiffMoMError(f"dmb_batch_create failed ({st})")
        self.h = h
        self.lanes = lanes

    def close(self):
        if self.h:
            self.lib.dmb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, surfaces, k: float, precision: str = "mixed", preconditioner: str = "lu",
              cutoff: float = math.inf, tol: float = 1e-6, maxiter: int = 300, precond_side: str = "left",
              quad_order: int = 3, eta0: float = ETA0_DEFAULT, return_currents: bool = False) -> BatchResult:
        if precision not in _PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}")
        if preconditioner not in EFIEDevice._PC_CODES:
            raise ValueError(f"unknown preconditioner {preconditioner!r}")
        side = {"left": nat.SIDE_LEFT, "right": nat.SIDE_RIGHT}.get(precond_side)
        if side is None:
            raise ValueError(f"Invalid precond_side: {precond_side} (expected :left or :right)")
        surfaces = list(surfaces)
        if not surfaces:
            raise ValueError("solve: need at least one surface")
        items = (nat.BatchItem * len(surfaces))()
        keep, outs = [], []
        for it, sf in zip(items, surfaces):
            m, r = sf.mesh, sf.rwg
            if r.mesh is not m:
                raise ValueError("RWG data was built for a different mesh")
            arrs = [np.ascontiguousarray(m.xyz, dtype=np.float64), np.ascontiguousarray(m.tri, dtype=np.int64)]
            arrs += [np.ascontiguousarray(a, dtype=np.int64)
                     for a in (r.tplus, r.tminus, r.evert, r.vplus_opp, r.vminus_opp)]
            arrs += [np.ascontiguousarray(a, dtype=np.float64) for a in (r.len, r.area_plus, r.area_minus)]
            zs = None
            if sf.zs is not None:
                zs = np.ascontiguousarray(np.broadcast_to(np.asarray(sf.zs, dtype=np.complex128),
                                                          (m.ntriangles,)))
            I = np.empty(r.nedges, dtype=np.complex128) if return_currents else None
            keep.append((arrs, zs, I))
            outs.append(I)
            it.xyz, it.tri = arrs[0].ctypes.data, arrs[1].ctypes.data
            it.nv, it.nt, it.n = m.nvertices, m.ntriangles, r.nedges
            it.tplus, it.tminus, it.evert, it.vplus_opp, it.vminus_opp = (a.ctypes.data for a in arrs[2:7])
            it.len, it.area_plus, it.area_minus = (a.ctypes.data for a in arrs[7:10])
            it.zs = zs.ctypes.data if zs is not None else None
            e = sf.excitation
            it.kvec[:] = [float(v) for v in e.k_vec]
            it.pol[:] = [float(v) for v in e.pol]
            it.E0 = float(e.E0)
            it.I_out = I.ctypes.data if I is not None else None
        p = nat.SolveParams()
        p.k, p.eta0, p.cutoff, p.tol = float(k), float(eta0), float(cutoff), float(tol)
        p.quad_order, p.precision = int(quad_order), _PRECISIONS[precision]
        p.precond_kind, p.precond_side, p.maxiter = EFIEDevice._PC_CODES[preconditioner], side, int(maxiter)
        dms = ctypes.c_double()
        st = self.lib.dmb_batch_solve(self.h, ctypes.byref(p), items, len(surfaces), ctypes.byref(dms))
        if st != nat.DMB_OK:
            msg = (self.lib.dmb_batch_last_error(self.h) or b"").decode()
            raise nat._EXC.get(st, nat.DiffMoMError)(msg)
        ams = ctypes.c_double()
        self.lib.dmb_batch_assembly_ms(self.h, ctypes.byref(ams))
        return BatchResult(sigma=np.array([it.sigma for it in items]),
                           gmres_iters=np.array([it.stats.niter for it in items]),
                           true_residual=np.array([it.stats.true_residual for it in items]),
                           latency_ms=np.array([it.latency_ms for it in items]),
                           solve_ms=np.array([it.solve_ms for it in items]),
                           device_ms=dms.value, N=np.array([it.n for it in items]),
                           currents=outs if return_currents else None, assembly_ms=ams.value)


def solve_surfaces(surfaces, freq_hz, lanes: int = 8, precision: str = "mixed", preconditioner: str = "lu",
                   nf_cutoff_lambda: float = math.inf, gmres_tol: float = 1e-6, gmres_maxiter: int = 300,
                   precond_side: str = "left", quad_order: int = 3, c0: float = C0_DEFAULT,
                   return_currents: bool = False, batch: SurfaceBatch | None = None) -> BatchResult:
    """solve_scattering (Workflow.jl:67-317) + backscatter_rcs for many
    independent surfaces (BatchSurface: mesh, rwg, plane wave, optional
    per-triangle impedance) in one call; see SurfaceBatch."""
    f = float(freq_hz)
    if not (math.isfinite(f) and f > 0):
        raise ValueError(f"solve_surfaces: freq_hz must be finite and positive, got {freq_hz}")
    k = _frequency_to_wavenumber(f, c0)
    b = batch or SurfaceBatch(lanes)
    try:
        return b.solve(surfaces, k, precision=precision, preconditioner=preconditioner,
                       cutoff=nf_cutoff_lambda * (c0 / f), tol=gmres_tol, maxiter=gmres_maxiter,
                       precond_side=precond_side, quad_order=quad_order, return_currents=return_currents)
    finally:
        if batch is None:
            b.close()


# ---------------------------------------------------------------------------
# far field / RCS
# ---------------------------------------------------------------------------
@dataclass
class SphGrid:
    rhat: np.ndarray   # (NO, 3)
    theta: np.ndarray
    phi: np.ndarray
    w: np.ndarray


def make_sph_grid(Ntheta: int, Nphi: int) -> SphGrid:
    """FarField.jl:216-277: midpoint grid in theta and phi."""
    if Ntheta <= 0 or Nphi <= 0:
        raise ValueError("Ntheta and Nphi must be positive")
    dth, dph = math.pi / Ntheta, 2 * math.pi / Nphi
    th = (np.arange(1, Ntheta + 1) - 0.5) * dth
    ph = (np.arange(1, Nphi + 1) - 0.5) * dph
    T, P = np.meshgrid(th, ph, indexing="ij")
    T, P = T.ravel(), P.ravel()
    rh = np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], axis=1)
    return SphGrid(rh, T, P, np.sin(T) * dth * dph)


def phi_cut_grid(phi: float, thetas_deg) -> SphGrid:
    th = np.deg2rad(np.asarray(thetas_deg, dtype=np.float64))
    rh = np.stack([np.sin(th) * math.cos(phi), np.sin(th) * math.sin(phi), np.cos(th)], axis=1)
    return SphGrid(rh, th, np.full(th.shape, phi), np.ones(th.shape))


def compute_farfield(device: EFIEDevice, grid: SphGrid, I, k=None, eta0=ETA0_DEFAULT, quad_order=3):
    """E_ff (3 x NO [x nrhs]) = G_mat * I on the device."""
    return device.farfield(grid.rhat, I, k=k, eta0=eta0, quad_order=quad_order)


def bistatic_rcs(E_ff: np.ndarray, E0: float = 1.0) -> np.ndarray:
    """Diagnostics.jl:460-474: sigma = 4 pi |E_inf|^2 / |E0|^2."""
    if E_ff.shape[0] != 3:
        raise nat.DimensionMismatch(f"E_ff has {E_ff.shape[0]} rows, expected 3")
    return 4 * math.pi * np.sum(np.abs(E_ff) ** 2, axis=0) / abs(E0) ** 2


def backscatter_rcs(E_ff: np.ndarray, grid: SphGrid, k_inc_hat, E0: float = 1.0):
    kh = np.asarray(k_inc_hat, dtype=np.float64)
    kh = kh / np.linalg.norm(kh)
    d = grid.rhat @ (-kh)
    idx = int(np.argmax(d))
    sig = bistatic_rcs(E_ff[:, idx:idx + 1], E0)[0]
    return dict(sigma=sig, index=idx, theta=grid.theta[idx], phi=grid.phi[idx],
                angular_error_deg=math.degrees(math.acos(max(-1.0, min(1.0, d[idx])))))
