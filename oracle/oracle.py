"""Python side of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads oracle/_build/libefie_oracle.so (the C restatement in efie_oracle.c) and
adds numpy restatements of the solver pieces:

* ``gmres``      -- Krylov.gmres semantics as called by solve_gmres
                    (IterativeSolve.jl:341-392): x0 = 0, no restart, modified
                    Gram-Schmidt Arnoldi, Givens rotations, rtol*||r0|| with
                    r0 = M b (left) or b (right/none).
* ``nearfield_matrix`` -- near-field extraction (NearFieldPreconditioner.jl:
                    247-369, 670-716) as a dense matrix with zeros outside.
* ``mie_bistatic_rcs_pec`` -- published Mie series for a PEC sphere
                    (Bohren & Huffman 1983, ch. 4), the physics check the
                    reference runs in Test 13 (src/postprocessing/Mie.jl).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
this module, as the checker.  Parity: pinned to the reference tests' golden
values (Tests 2, 44, 45) and physics gate (Test 13); entrywise Z parity with a
live Julia run is unpinned (Julia is absent).
"""
from __future__ import annotations

import ctypes
import math
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libefie_oracle.so"
SRC = HERE / "efie_oracle.c"

_D = ctypes.c_double
_L = ctypes.c_int64
_I = ctypes.c_int
_P = ctypes.c_void_p
_DP = ctypes.POINTER(ctypes.c_double)
_LP = ctypes.POINTER(ctypes.c_int64)


def build(force: bool = False) -> Path:
    """Compile the oracle (gcc, OpenMP, no FMA contraction)."""
    if LIB.exists() and not force and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    LIB.parent.mkdir(exist_ok=True)
    subprocess.run(["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared", "-std=c11",
                    "-o", str(LIB), str(SRC), "-lm"], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB))
        L.orc_cache_build.restype = _P
        L.orc_cache_build.argtypes = [_DP, _L, _LP, _L, _L, _LP, _LP, _LP, _LP, _DP, _DP, _DP, _I]
        L.orc_cache_free.argtypes = [_P]
        L.orc_assemble_z.argtypes = [_P, _D, _D, _DP, _I]
        L.orc_max_threads.argtypes = []
        L.orc_max_threads.restype = ctypes.c_int
        L.orc_assemble_rows.argtypes = [_P, _D, _D, _L, _L, _DP, _I]
        L.orc_efie_entries.argtypes = [_P, _D, _D, _LP, _LP, _L, _DP]
        L.orc_plane_wave_rhs.argtypes = [_P, _DP, _D, _DP, _DP]
        L.orc_dipole_rhs.argtypes = [_P, _DP, _DP, _I, _D, _DP]
        L.orc_dipole_field.argtypes = [_DP, _L, _DP, _DP, _I, _D, _DP]
        L.orc_pattern_rhs.argtypes = [_P, _I, _DP, _I, _DP, _DP, _DP, _D, _DP, _I, _DP]
        L.orc_pattern_field.argtypes = [_DP, _L, _I, _DP, _I, _DP, _DP, _DP, _D, _DP, _I, _DP]
        L.orc_apply_impedance.argtypes = [_P, _DP, _DP]
        L.orc_gradient_impedance.argtypes = [_P, _L, _DP, _DP, ctypes.POINTER(ctypes.c_int), _L, _I, _DP]
        L.orc_radiation_vectors.argtypes = [_P, _DP, _L, _D, _D, _DP]
        L.orc_adjacent_pair_count.restype = _L
        L.orc_adjacent_pair_count.argtypes = [_P]
        L.orc_cache_quad_points.argtypes = [_P, _DP, _DP, _DP]
        L.orc_analytic_1overR.argtypes = [_DP, _DP, _DP, _DP, _DP]
        L.orc_analytic_1overR_unchecked.restype = _D
        L.orc_analytic_1overR_unchecked.argtypes = [_DP, _DP, _DP, _DP]
        L.orc_greens.argtypes = [_DP, _DP, _D, _DP]
        L.orc_greens_smooth.argtypes = [_DP, _DP, _D, _DP]
        L.orc_triangle_area.restype = _D
        L.orc_triangle_area.argtypes = [_DP, _DP, _DP]
        L.orc_fallback_count.restype = ctypes.c_long
        L.orc_nearfield_mask.argtypes = [_DP, _L, _D, ctypes.POINTER(ctypes.c_uint8)]
        L.orc_quad_rule.argtypes = [_I, _DP, _DP, _DP]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_DP)


def _l(a):
    return a.ctypes.data_as(_LP)


def _v3(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(3))


def greens(r, rp, k) -> complex:
    out = np.zeros(2)
    lib().orc_greens(_d(_v3(r)), _d(_v3(rp)), float(k), _d(out))
    return complex(out[0], out[1])


def greens_smooth(r, rp, k) -> complex:
    out = np.zeros(2)
    lib().orc_greens_smooth(_d(_v3(r)), _d(_v3(rp)), float(k), _d(out))
    return complex(out[0], out[1])


def analytical_integral_1overR(P, V1, V2, V3) -> float:
    out = np.zeros(1)
    st = lib().orc_analytic_1overR(_d(_v3(P)), _d(_v3(V1)), _d(_v3(V2)), _d(_v3(V3)), _d(out))
    if st != 0:
        raise ValueError("static-integral geometry is degenerate or non-finite")
    return float(out[0])


def tri_quad_rule(order: int):
    x1, x2, w = np.zeros(7), np.zeros(7), np.zeros(7)
    n = lib().orc_quad_rule(order, _d(x1), _d(x2), _d(w))
    if n < 0:
        raise ValueError(f"Unsupported quadrature order {order}")
    return np.stack([x1[:n], x2[:n]], axis=1), w[:n]


class OracleCache:
    """EFIEApplyCache restatement (EFIE.jl:332-398) for one mesh + RWG set."""

    def __init__(self, mesh, rwg, quad_order: int = 3):
        self.mesh, self.rwg = mesh, rwg
        self._keep = [np.ascontiguousarray(mesh.xyz, dtype=np.float64),
                      np.ascontiguousarray(mesh.tri, dtype=np.int64)]
        self._r = [np.ascontiguousarray(getattr(rwg, f), dtype=t) for f, t in (
            ("tplus", np.int64), ("tminus", np.int64), ("vplus_opp", np.int64),
            ("vminus_opp", np.int64), ("len", np.float64), ("area_plus", np.float64),
            ("area_minus", np.float64))]
        tp, tm, vp, vm, ln, ap, am = self._r
        self.N = rwg.nedges
        self.nq = len(tri_quad_rule(quad_order)[1])
        self.h = lib().orc_cache_build(_d(self._keep[0]), mesh.nvertices, _l(self._keep[1]),
                                       mesh.ntriangles, self.N, _l(tp), _l(tm), _l(vp), _l(vm),
                                       _d(ln), _d(ap), _d(am), quad_order)
        if not self.h:
            raise ValueError(f"Unsupported quadrature order {quad_order}")

    def __del__(self):
        try:
            lib().orc_cache_free(self.h)
        except Exception:
            pass

    def adjacent_pair_count(self) -> int:
        return int(lib().orc_adjacent_pair_count(self.h))

    def quad_points(self):
        nt = self.mesh.ntriangles
        qp, qph, ar = np.zeros((nt, self.nq, 3)), np.zeros((nt, 7, 3)), np.zeros(nt)
        lib().orc_cache_quad_points(self.h, _d(qp), _d(qph), _d(ar))
        return qp, qph, ar

    def assemble_z(self, k, eta0=376.730313668, nthreads=0) -> np.ndarray:
        Z = np.zeros((self.N, self.N), dtype=np.complex128, order="F")
        lib().orc_assemble_z(self.h, float(k), float(eta0), _d(Z), int(nthreads))
        return Z

    def assemble_rows(self, k, m0, m1, eta0=376.730313668, nthreads=0) -> np.ndarray:
        rows = np.zeros((m1 - m0, self.N), dtype=np.complex128)
        lib().orc_assemble_rows(self.h, float(k), float(eta0), m0, m1, _d(rows),
                                int(nthreads))
        return rows

    def entries(self, k, m, n, eta0=376.730313668) -> np.ndarray:
        m = np.ascontiguousarray(m, dtype=np.int64)
        n = np.ascontiguousarray(n, dtype=np.int64)
        out = np.zeros(m.size, dtype=np.complex128)
        lib().orc_efie_entries(self.h, float(k), float(eta0), _l(m), _l(n), m.size,
                               _d(out))
        return out

    def plane_wave_rhs(self, k_vec, E0, pol) -> np.ndarray:
        v = np.zeros(self.N, dtype=np.complex128)
        lib().orc_plane_wave_rhs(self.h, _d(_v3(k_vec)), float(E0), _d(_v3(pol)),
                                 _d(v))
        return v

    def dipole_rhs(self, position, moment, dipole_type="electric", frequency=1e9) -> np.ndarray:
        """assemble_dipole (Excitation.jl:2924-2953); loop: magnetic dipole of
        moment I pi a^2 n (Excitation.jl:936-942, 2187-2198)."""
        m = np.asarray(moment, dtype=np.complex128)
        mm = np.ascontiguousarray(np.stack([m.real, m.imag], 1).ravel())
        v = np.zeros(self.N, dtype=np.complex128)
        lib().orc_dipole_rhs(self.h, _d(_v3(position)), _d(mm), 1 if dipole_type == "magnetic" else 0,
                             float(frequency), _d(v))
        return v

    def pattern_rhs(self, theta, phi, Ftheta, Fphi, frequency, phase_center=(0.0, 0.0, 0.0),
                    conj_convention=False) -> np.ndarray:
        """assemble_pattern_feed (Excitation.jl:3044-3071); angles in radians,
        F matrices (ntheta, nphi); conj_convention for exp(-i omega t) data."""
        a = _pattern_args(theta, phi, Ftheta, Fphi)
        v = np.zeros(self.N, dtype=np.complex128)
        lib().orc_pattern_rhs(self.h, a[0], _d(a[1]), a[2], _d(a[3]), _d(a[4]), _d(a[5]), float(frequency),
                              _d(_v3(phase_center)), 1 if conj_convention else 0, _d(v))
        return v

    def gradient_impedance(self, I, lam, tri_patch, P, reactive=False) -> np.ndarray:
        """gradient_impedance (Adjoint.jl:1081-1119) for per-triangle patch ids
        (0-based); I, lam (N,) or (N, R); returns (P,) or (P, R)."""
        Ia = np.asfortranarray(np.asarray(I, dtype=np.complex128).reshape(self.N, -1))
        La = np.asfortranarray(np.asarray(lam, dtype=np.complex128).reshape(self.N, -1))
        tp = np.ascontiguousarray(tri_patch, dtype=np.int32)
        R = Ia.shape[1]
        g = np.zeros((int(P), R), dtype=np.float64, order="F")
        rc = lib().orc_gradient_impedance(self.h, R, _d(Ia), _d(La), tp.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                          int(P), 1 if reactive else 0, _d(g))
        if rc != 0:
            raise MemoryError("oracle gradient: allocation failed")
        return g[:, 0] if np.asarray(I).ndim == 1 else g

    def apply_impedance(self, Z: np.ndarray, zs) -> np.ndarray:
        Zc = np.asfortranarray(Z.copy())
        zsa = np.ascontiguousarray(np.broadcast_to(np.asarray(zs, dtype=np.complex128),
                                                   (self.mesh.ntriangles,)))
        lib().orc_apply_impedance(self.h, _d(zsa), _d(Zc))
        return Zc

    def radiation_vectors(self, rhat, k, eta0=376.730313668) -> np.ndarray:
        rh = np.ascontiguousarray(np.atleast_2d(rhat), dtype=np.float64)
        NO = rh.shape[0]
        G = np.zeros((3 * NO, self.N), dtype=np.complex128, order="F")
        lib().orc_radiation_vectors(self.h, _d(rh), NO, float(k), float(eta0), _d(G))
        return G


def dipole_field(points, position, moment, dipole_type="electric", frequency=1e9) -> np.ndarray:
    """_dipole_incident_field_unchecked (Excitation.jl:2131-2185) at points (n x 3)."""
    r = np.ascontiguousarray(np.atleast_2d(points), dtype=np.float64)
    m = np.asarray(moment, dtype=np.complex128)
    mm = np.ascontiguousarray(np.stack([m.real, m.imag], 1).ravel())
    E = np.zeros((r.shape[0], 3), dtype=np.complex128)
    lib().orc_dipole_field(_d(r), r.shape[0], _d(_v3(position)), _d(mm), 1 if dipole_type == "magnetic" else 0,
                           float(frequency), _d(E))
    return E


def _pattern_args(theta, phi, Ftheta, Fphi):
    th = np.ascontiguousarray(theta, dtype=np.float64)
    ph = np.ascontiguousarray(phi, dtype=np.float64)
    ft = np.asfortranarray(np.asarray(Ftheta, dtype=np.complex128).reshape(th.size, ph.size))
    fp = np.asfortranarray(np.asarray(Fphi, dtype=np.complex128).reshape(th.size, ph.size))
    # column-major complex matrices as interleaved doubles
    ftv = np.ascontiguousarray(np.stack([ft.real.ravel(order="F"), ft.imag.ravel(order="F")], 1).ravel())
    fpv = np.ascontiguousarray(np.stack([fp.real.ravel(order="F"), fp.imag.ravel(order="F")], 1).ravel())
    return th.size, th, ph.size, ph, ftv, fpv


def pattern_field(points, theta, phi, Ftheta, Fphi, frequency, phase_center=(0.0, 0.0, 0.0),
                  conj_convention=False) -> np.ndarray:
    """_pattern_feed_field_unchecked (Excitation.jl:1417-1460) at points (n x 3)."""
    r = np.ascontiguousarray(np.atleast_2d(points), dtype=np.float64)
    a = _pattern_args(theta, phi, Ftheta, Fphi)
    E = np.zeros((r.shape[0], 3), dtype=np.complex128)
    lib().orc_pattern_field(_d(r), r.shape[0], a[0], _d(a[1]), a[2], _d(a[3]), _d(a[4]), _d(a[5]),
                            float(frequency), _d(_v3(phase_center)), 1 if conj_convention else 0, _d(E))
    return E


def fallback_count() -> int:
    return int(lib().orc_fallback_count())


def nearfield_matrix(Z: np.ndarray, centers: np.ndarray, cutoff: float) -> np.ndarray:
    N = Z.shape[0]
    mask = np.zeros((N, N), dtype=np.uint8, order="F")
    c = np.ascontiguousarray(centers, dtype=np.float64)
    lib().orc_nearfield_mask(_d(c), N, float(cutoff), mask.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
    return np.where(mask.astype(bool), Z, 0)


def gmres(A, b, M=None, side="left", rtol=1e-8, itmax=200):
    """Krylov.gmres restatement (no restart, MGS, Givens).  A, M: callables or
    matrices (M applies the inverse preconditioner).  Returns (x, niter, solved)."""
    Aop = (lambda v: A @ v)
    Mop = (lambda v: v) if M is None else ((lambda v: M @ v) if not callable(M) else M)
    left = M is not None and side == "left"
    right = M is not None and side == "right"
    b = np.asarray(b, dtype=np.complex128)
    r0 = Mop(b) if left else b.copy()
    beta = np.linalg.norm(r0)
    if beta == 0:
        return np.zeros_like(b), 0, True
    eps = rtol * beta
    n = b.size
    V = np.zeros((itmax + 1, n), dtype=np.complex128)
    H = np.zeros((itmax + 1, itmax), dtype=np.complex128)
    cs = np.zeros(itmax)
    sn = np.zeros(itmax, dtype=np.complex128)
    g = np.zeros(itmax + 1, dtype=np.complex128)
    g[0] = beta
    V[0] = r0 / beta
    k = 0
    solved = False
    for j in range(itmax):
        w = V[j]
        if right:
            w = Mop(w)
        w = Aop(w)
        if left:
            w = Mop(w)
        for i in range(j + 1):
            H[i, j] = np.vdot(V[i], w)
            w = w - H[i, j] * V[i]
        H[j + 1, j] = np.linalg.norm(w)
        if H[j + 1, j] != 0:
            V[j + 1] = w / H[j + 1, j]
        for i in range(j):
            a, bb = H[i, j], H[i + 1, j]
            H[i, j] = cs[i] * a + sn[i] * bb
            H[i + 1, j] = cs[i] * bb - np.conj(sn[i]) * a
        a, bb = H[j, j], H[j + 1, j]
        na, nb = abs(a), abs(bb)
        if nb == 0:
            c, s, rho = 1.0, 0.0, a
        elif na == 0:
            c, s, rho = 0.0, np.conj(bb) / nb, nb
        else:
            t = math.hypot(na, nb)
            sa = a / na
            c, s, rho = na / t, sa * np.conj(bb) / t, sa * t
        cs[j], sn[j] = c, s
        H[j, j], H[j + 1, j] = rho, 0
        g[j + 1] = -np.conj(s) * g[j]
        g[j] = c * g[j]
        k = j + 1
        if abs(g[j + 1]) <= eps:
            solved = True
            break
    y = np.linalg.solve(np.triu(H[:k, :k]), g[:k]) if k else np.zeros(0)
    x = V[:k].T @ y
    if right:
        x = Mop(x)
    return x, k, solved


# ---------------------------------------------------------------------------
# Mie series, PEC sphere (Bohren & Huffman 1983, eqs. 4.53, 4.74; PEC limit)
# ---------------------------------------------------------------------------
def _mie_pec_coeffs(x: float, nmax: int):
    from scipy.special import spherical_jn, spherical_yn
    n = np.arange(1, nmax + 1)
    jn = spherical_jn(n, x)
    yn = spherical_yn(n, x)
    jn1 = spherical_jn(n - 1, x)
    yn1 = spherical_yn(n - 1, x)
    psi = x * jn
    xi = x * (jn + 1j * yn)
    dpsi = x * jn1 - n * jn
    dxi = x * (jn1 + 1j * yn1) - n * (jn + 1j * yn)
    a = dpsi / dxi
    b = psi / xi
    return n, a, b


def mie_s1s2_pec(x: float, mu: float, nmax=None):
    nmax = nmax or int(x + 4 * x ** (1 / 3) + 2)
    n, a, b = _mie_pec_coeffs(x, nmax)
    pi_n = np.zeros(nmax + 1)
    tau_n = np.zeros(nmax + 1)
    pi_n[1] = 1.0
    tau_n[1] = mu
    if nmax >= 2:
        pi_n[2] = 3 * mu
        tau_n[2] = 2 * mu * pi_n[2] - 3 * pi_n[1]
    for k in range(3, nmax + 1):
        pi_n[k] = ((2 * k - 1) * mu * pi_n[k - 1] - k * pi_n[k - 2]) / (k - 1)
        tau_n[k] = k * mu * pi_n[k] - (k + 1) * pi_n[k - 1]
    f = (2 * n + 1) / (n * (n + 1))
    S1 = np.sum(f * (a * pi_n[1:] + b * tau_n[1:]))
    S2 = np.sum(f * (a * tau_n[1:] + b * pi_n[1:]))
    return S1, S2


def mie_bistatic_rcs_pec(k, a, k_inc_hat, pol_inc, rhat):
    kh = np.asarray(k_inc_hat, float) / np.linalg.norm(k_inc_hat)
    ph = np.asarray(pol_inc, float) / np.linalg.norm(pol_inc)
    rh = np.asarray(rhat, float) / np.linalg.norm(rhat)
    mu = float(np.clip(kh @ rh, -1, 1))
    e_perp = np.cross(kh, rh)
    if np.linalg.norm(e_perp) < 1e-12:
        t = np.array([1.0, 0, 0]) if abs(kh[0]) < 0.9 else np.array([0, 1.0, 0])
        e_perp = np.cross(kh, t)
    e_perp /= np.linalg.norm(e_perp)
    e_par_i = np.cross(e_perp, kh)
    e_par_i /= np.linalg.norm(e_par_i)
    c_perp = ph @ e_perp
    c_para = ph @ e_par_i
    S1, S2 = mie_s1s2_pec(k * a, mu)
    return 4 * math.pi / k ** 2 * (abs(S1 * c_perp) ** 2 + abs(S2 * c_para) ** 2)


def max_threads() -> int:
    """Threads the oracle's OpenMP loops can use (1 when built serial)."""
    return int(lib().orc_max_threads())
