// dmb_excitation.cu -- plane-wave right-hand sides, far field, and the
// matrix-free operator.
//
//   * assemble_plane_wave (Excitation.jl:2866-2896): v_n = sum over T+/T- and
//     quadrature points of -2 w_q A_t conj(f_n) . E0 pol exp(-i k.r_q)
//   * radiation_vectors + compute_farfield (FarField.jl:425-611):
//     E(rh) = i k eta0/(4 pi) sum_n I_n sum rh x (rh x f_n) w 2A exp(+i k rh.r')
//   * MatrixFreeEFIEOperator mul! (EFIE.jl:867-909): Z x recomputed from the
//     geometry without an N^2 store -- far triangle pairs on the fly in
//     triangle-slot space, near records precomputed once.
#include <algorithm>
#include <cmath>

#include "dmb_device.cuh"
#include "dmb_internal.h"

namespace {

unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// V (N x R column-major)
__global__ void k_plane_wave(int64_t N, int64_t R, const TriCache *__restrict__ tc, const int *__restrict__ rslot,
                             int nq, const double *__restrict__ wq, const double *__restrict__ kv,
                             const double *__restrict__ E0, const double *__restrict__ pol,
                             double2 *__restrict__ V) {
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= N * R) return;
  int64_t r = idx / N, n = idx % N;
  double k0 = kv[3 * r], k1 = kv[3 * r + 1], k2 = kv[3 * r + 2];
  double e0 = E0[r];
  double p0 = pol[3 * r] * e0, p1 = pol[3 * r + 1] * e0, p2 = pol[3 * r + 2] * e0;
  double2 acc = make_double2(0, 0);
  for (int s = 0; s < 2; s++) {
    int sl = rslot[2 * n + s];
    const TriCache &T = tc[sl / 3];
    int i = sl % 3;
    for (int q = 0; q < nq; q++) {
      double f0 = T.s[i] * (T.qp[q][0] - T.p[i][0]);
      double f1 = T.s[i] * (T.qp[q][1] - T.p[i][1]);
      double f2 = T.s[i] * (T.qp[q][2] - T.p[i][2]);
      double arg = k0 * T.qp[q][0] + k1 * T.qp[q][1] + k2 * T.qp[q][2];
      double sn, cs;
      sincos(arg, &sn, &cs);
      // E = pol*E0*(cos arg - i sin arg); inner = f . E
      double fe = f0 * p0 + f1 * p1 + f2 * p2;
      double2 ip = make_double2(fe * cs, -fe * sn);
      double2 ap = cscale(ip, T.area);
      acc = cadd(acc, cscale(ap, -(2 * wq[q])));
    }
  }
  V[idx] = acc;
}

// Dipole sources (electric or magnetic; a loop is the magnetic dipole of
// moment I pi a^2 n): field _dipole_incident_field_unchecked
// (Excitation.jl:2131-2185) at every quadrature point, folded with the RWG
// basis as assemble_dipole (Excitation.jl:2924-2953).  V (N x R column-major).
__device__ __forceinline__ double dop(double a, double b, double c, double d) {
  const double cd = c * d;
  return fma(a, b, -cd) + fma(-c, d, cd);
}
// complex a x real b
__device__ __forceinline__ void ccross(const double2 *a, const double *b, double2 *o) {
  o[0] = make_double2(dop(a[1].x, b[2], a[2].x, b[1]), dop(a[1].y, b[2], a[2].y, b[1]));
  o[1] = make_double2(dop(a[2].x, b[0], a[0].x, b[2]), dop(a[2].y, b[0], a[0].y, b[2]));
  o[2] = make_double2(dop(a[0].x, b[1], a[1].x, b[0]), dop(a[0].y, b[1], a[1].y, b[0]));
}

__device__ void dipole_field(const double *r, const double *pos, const double2 *p, int magnetic, double k,
                             double eta0, double eps0, double2 *E) {
  double d[3] = {r[0] - pos[0], r[1] - pos[1], r[2] - pos[2]};
  const double R = hypot(hypot(d[0], d[1]), d[2]);
  if (R == 0.0) {
    E[0] = E[1] = E[2] = make_double2(0, 0);
    return;
  }
  // direction rescaled by a power of two (largest component in [1, 2)) as
  // _source_power_of_two_scaled_direction (Excitation.jl:632-646): the
  // formulas only use d through d/|d| and d d^T/|d|^2
  {
    int e = -1 << 30;
    for (int i = 0; i < 3; i++)
      if (d[i] != 0.0) e = max(e, ilogb(d[i]));
    for (int i = 0; i < 3; i++) d[i] = scalbn(d[i], -e);
  }
  const double dn2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  double sn, cs;
  sincos(-k * R, &sn, &cs);
  const double2 phase = make_double2(cs, sn);
  if (!magnetic) {
    double2 pxd[3], dxp[3], t1[3];
    ccross(p, d, pxd);
    for (int i = 0; i < 3; i++) dxp[i] = make_double2(-pxd[i].x, -pxd[i].y);
    ccross(dxp, d, t1);
    double2 dp = make_double2(0, 0);
    for (int i = 0; i < 3; i++) dp = cadd(dp, cscale(p[i], d[i]));
    const double2 fac = make_double2(1.0 / (R * R), k / R);
    const double inv = 1.0 / (4.0 * 3.14159265358979323846 * eps0 * R);
    for (int i = 0; i < 3; i++) {
      const double2 term1 = cscale(cscale(t1[i], 1.0 / dn2), k * k);
      const double2 radial = cscale(cscale(dp, d[i]), 1.0 / dn2);
      const double2 term2 = cmul(csub(cscale(radial, 3.0), p[i]), fac);
      E[i] = cscale(cmul(cadd(term1, term2), phase), inv);
    }
  } else {
    const double2 rf = make_double2((eta0 / (4.0 * 3.14159265358979323846)) * (k * k / R),
                                    -(eta0 / (4.0 * 3.14159265358979323846)) * (k / (R * R)));
    const double2 pf = cmul(rf, phase);
    double2 ang[3];
    ccross(p, d, ang);
    const double nd = sqrt(dn2);
    for (int i = 0; i < 3; i++) E[i] = cmul(pf, cscale(ang[i], 1.0 / nd));
  }
}

__global__ void k_dipole_rhs(int64_t N, int64_t R, const TriCache *__restrict__ tc, const int *__restrict__ rslot,
                             int nq, const double *__restrict__ wq, const double *__restrict__ pos,
                             const double *__restrict__ mom, const int *__restrict__ magnetic,
                             const double *__restrict__ freq, double2 *__restrict__ V) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= N * R) return;
  const int64_t r = idx / N, n = idx % N;
  const double eps0 = 8.854187817e-12, mu0 = 4.0 * 3.14159265358979323846 * 1e-7;
  const double eta0 = sqrt(mu0 / eps0), c0 = 1.0 / sqrt(eps0 * mu0);
  const double k = (2.0 * 3.14159265358979323846 * freq[r]) / c0;
  const double2 p[3] = {make_double2(mom[6 * r], mom[6 * r + 1]), make_double2(mom[6 * r + 2], mom[6 * r + 3]),
                        make_double2(mom[6 * r + 4], mom[6 * r + 5])};
  double2 acc = make_double2(0, 0);
  for (int s = 0; s < 2; s++) {
    const int sl = rslot[2 * n + s];
    const TriCache &T = tc[sl / 3];
    const int i = sl % 3;
    for (int q = 0; q < nq; q++) {
      const double f0 = T.s[i] * (T.qp[q][0] - T.p[i][0]);
      const double f1 = T.s[i] * (T.qp[q][1] - T.p[i][1]);
      const double f2 = T.s[i] * (T.qp[q][2] - T.p[i][2]);
      double2 E[3];
      dipole_field(T.qp[q], pos + 3 * r, p, magnetic[r], k, eta0, eps0, E);
      const double2 ip = cadd(cadd(cscale(E[0], f0), cscale(E[1], f1)), cscale(E[2], f2));
      const double2 ap = cscale(ip, T.area);
      acc = cadd(acc, cscale(ap, -(2 * wq[q])));
    }
  }
  V[idx] = acc;
}

// Pattern feed (Excitation.jl:1170-1340, 1417-1460): E(r) = exp(-ikR)/R
// (F_theta e_theta + F_phi e_phi) of r - phase_center, F bilinear in
// (theta, phi) on the grid -- theta clamped to its range, phi periodic with
// the interval from the last sample back to the first + 2 pi -- and conjugated
// for exp(-i omega t) data.  F matrices column-major (ntheta x nphi).  Folded
// with the RWG basis as assemble_pattern_feed (Excitation.jl:3044-3071).
struct PatternDev {
  int nth, nph;
  const double *th, *ph;
  const double2 *Ft, *Fp;
  double k, pc[3];
  int conj;
};

// largest i with g[i] <= x (g strictly increasing, x >= g[0])
__device__ int pat_search_last(const double *g, int n, double x) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (g[mid] <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ double2 pat_bilinear(const double2 *M, int nth, int it, int jt, double tt, int ip, int jp, double tp) {
  const double2 c00 = M[it + (int64_t)ip * nth];
  if (it == jt && ip == jp) return c00;
  if (it == jt) return cadd(cscale(c00, 1 - tp), cscale(M[it + (int64_t)jp * nth], tp));
  if (ip == jp) return cadd(cscale(c00, 1 - tt), cscale(M[jt + (int64_t)ip * nth], tt));
  const double2 c10 = M[jt + (int64_t)ip * nth], c01 = M[it + (int64_t)jp * nth], c11 = M[jt + (int64_t)jp * nth];
  return cadd(cadd(cadd(cscale(c00, (1 - tt) * (1 - tp)), cscale(c10, tt * (1 - tp))), cscale(c01, (1 - tt) * tp)),
              cscale(c11, tt * tp));
}

__device__ void pattern_field(const double *r, const PatternDev &P, double2 *E) {
  const double two_pi = 2.0 * 3.14159265358979323846;
  const double d[3] = {r[0] - P.pc[0], r[1] - P.pc[1], r[2] - P.pc[2]};
  const double R = hypot(hypot(d[0], d[1]), d[2]);
  if (R == 0.0) {
    E[0] = E[1] = E[2] = make_double2(0, 0);
    return;
  }
  const double th = acos(fmin(1.0, fmax(-1.0, d[2] / R)));
  double ph = atan2(d[1], d[0]);
  if (ph < 0) ph += two_pi;
  double st, ct, sp, cp;
  sincos(th, &st, &ct);
  sincos(ph, &sp, &cp);
  const double et[3] = {ct * cp, ct * sp, -st}, ep[3] = {-sp, cp, 0.0};
  // theta: clamped
  int it, jt;
  double tt;
  if (th <= P.th[0]) {
    it = jt = 0;
    tt = 0.0;
  } else if (th >= P.th[P.nth - 1]) {
    it = jt = P.nth - 1;
    tt = 0.0;
  } else {
    it = min(pat_search_last(P.th, P.nth, th), P.nth - 2);
    jt = it + 1;
    tt = (th - P.th[it]) / (P.th[jt] - P.th[it]);
  }
  // phi: periodic (floored modulo)
  double m = fmod(ph - P.ph[0], two_pi);
  if (m != 0.0 && m < 0.0) m += two_pi;
  const double w = m + P.ph[0];
  int ip, jp;
  double tp;
  const int n = P.nph;
  if (w <= P.ph[n - 1]) {
    const int a = pat_search_last(P.ph, n, w);
    if (a == n - 1) {
      ip = n - 1;
      jp = 0;
      tp = (w - P.ph[n - 1]) / (P.ph[0] + two_pi - P.ph[n - 1]);
    } else {
      ip = a;
      jp = a + 1;
      tp = (w - P.ph[a]) / (P.ph[a + 1] - P.ph[a]);
    }
  } else {
    ip = n - 1;
    jp = 0;
    tp = (w - P.ph[n - 1]) / (P.ph[0] + two_pi - P.ph[n - 1]);
  }
  double2 Ft = pat_bilinear(P.Ft, P.nth, it, jt, tt, ip, jp, tp);
  double2 Fp = pat_bilinear(P.Fp, P.nth, it, jt, tt, ip, jp, tp);
  if (P.conj) {
    Ft = cconj(Ft);
    Fp = cconj(Fp);
  }
  double sn, cs;
  sincos(-P.k * R, &sn, &cs);
  const double2 phase = make_double2(cs, sn);
  for (int a = 0; a < 3; a++)
    E[a] = cmul(cscale(cadd(cscale(Ft, et[a]), cscale(Fp, ep[a])), 1.0 / R), phase);
}

__global__ void k_pattern_rhs(int64_t N, const TriCache *__restrict__ tc, const int *__restrict__ rslot, int nq,
                              const double *__restrict__ wq, PatternDev P, double2 *__restrict__ V) {
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  double2 acc = make_double2(0, 0);
  for (int s = 0; s < 2; s++) {
    const int sl = rslot[2 * n + s];
    const TriCache &T = tc[sl / 3];
    const int i = sl % 3;
    for (int q = 0; q < nq; q++) {
      const double f0 = T.s[i] * (T.qp[q][0] - T.p[i][0]);
      const double f1 = T.s[i] * (T.qp[q][1] - T.p[i][1]);
      const double f2 = T.s[i] * (T.qp[q][2] - T.p[i][2]);
      double2 E[3];
      pattern_field(T.qp[q], P, E);
      const double2 ip = cadd(cadd(cscale(E[0], f0), cscale(E[1], f1)), cscale(E[2], f2));
      acc = cadd(acc, cscale(cscale(ip, T.area), -(2 * wq[q])));
    }
  }
  V[n] = acc;
}

// radiation matrix G (3*NO x N, row-major) for directions rh
__global__ void k_radiation(int64_t N, int64_t NO, const TriCache *__restrict__ tc, const int *__restrict__ rslot,
                            int nq, const double *__restrict__ wq, const double *__restrict__ rh, double k,
                            double eta0, double2 *__restrict__ G) {
  int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t q = blockIdx.y;
  if (n >= N) return;
  double r0 = rh[3 * q], r1 = rh[3 * q + 1], r2 = rh[3 * q + 2];
  double rn2 = r0 * r0 + r1 * r1 + r2 * r2;
  double2 c0 = make_double2(0, 0), c1 = c0, c2 = c0;
  for (int s = 0; s < 2; s++) {
    int sl = rslot[2 * n + s];
    const TriCache &T = tc[sl / 3];
    int i = sl % 3;
    for (int qs = 0; qs < nq; qs++) {
      double f0 = T.s[i] * (T.qp[qs][0] - T.p[i][0]);
      double f1 = T.s[i] * (T.qp[qs][1] - T.p[i][1]);
      double f2 = T.s[i] * (T.qp[qs][2] - T.p[i][2]);
      double wt = wq[qs] * 2 * T.area;
      double arg = k * (r0 * T.qp[qs][0] + r1 * T.qp[qs][1] + r2 * T.qp[qs][2]);
      double sn, cs;
      sincos(arg, &sn, &cs);
      double2 ph = make_double2(wt * cs, wt * sn);
      c0 = cadd(c0, cscale(ph, f0));
      c1 = cadd(c1, cscale(ph, f1));
      c2 = cadd(c2, cscale(ph, f2));
    }
  }
  // rh x (rh x C) / |rh|^2 = (rh (rh.C) - C |rh|^2) / |rh|^2
  double2 d = cadd(cadd(cscale(c0, r0), cscale(c1, r1)), cscale(c2, r2));
  double2 v0 = cscale(csub(cscale(d, r0), cscale(c0, rn2)), 1.0 / rn2);
  double2 v1 = cscale(csub(cscale(d, r1), cscale(c1, rn2)), 1.0 / rn2);
  double2 v2 = cscale(csub(cscale(d, r2), cscale(c2, rn2)), 1.0 / rn2);
  double2 pref = make_double2(0, k * eta0 * DMB_INV_FOUR_PI);
  G[(3 * q + 0) * N + n] = cmul(pref, v0);
  G[(3 * q + 1) * N + n] = cmul(pref, v1);
  G[(3 * q + 2) * N + n] = cmul(pref, v2);
}

// Monostatic far field: for incidence r the field of current column I_r in
// the direction -k_hat_r (one CTA per incidence, block reduction over RWGs),
// E (3 complex per r) and sigma_r = 4 pi |E|^2 / |E0_r|^2 (Diagnostics.jl:460-474).
__global__ void __launch_bounds__(256) k_monostatic(int64_t N, const TriCache *__restrict__ tc,
                                                    const int *__restrict__ rslot, int nq,
                                                    const double *__restrict__ wq, const double *__restrict__ kv,
                                                    const double *__restrict__ E0s, double k, double eta0,
                                                    const double2 *__restrict__ I, double2 *__restrict__ E,
                                                    double *__restrict__ sigma) {
  __shared__ double2 red[3][8];
  const int64_t r = blockIdx.x;
  const double kx = kv[3 * r], ky = kv[3 * r + 1], kz = kv[3 * r + 2];
  const double kn = sqrt(kx * kx + ky * ky + kz * kz);
  const double r0 = -kx / kn, r1 = -ky / kn, r2 = -kz / kn;
  double2 c0 = make_double2(0, 0), c1 = c0, c2 = c0;
  const double2 *Ir = I + r * N;
  for (int64_t n = threadIdx.x; n < N; n += blockDim.x) {
    const double2 in = Ir[n];
    for (int s = 0; s < 2; s++) {
      const int sl = rslot[2 * n + s];
      const TriCache &T = tc[sl / 3];
      const int i = sl % 3;
      for (int qs = 0; qs < nq; qs++) {
        const double wt = wq[qs] * 2 * T.area * T.s[i];
        const double arg = k * (r0 * T.qp[qs][0] + r1 * T.qp[qs][1] + r2 * T.qp[qs][2]);
        double sn, cs;
        sincos(arg, &sn, &cs);
        const double2 ph = cmul(make_double2(wt * cs, wt * sn), in);
        c0 = cadd(c0, cscale(ph, T.qp[qs][0] - T.p[i][0]));
        c1 = cadd(c1, cscale(ph, T.qp[qs][1] - T.p[i][1]));
        c2 = cadd(c2, cscale(ph, T.qp[qs][2] - T.p[i][2]));
      }
    }
  }
  c0 = warp_sum2(c0);
  c1 = warp_sum2(c1);
  c2 = warp_sum2(c2);
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][w] = c0;
    red[1][w] = c1;
    red[2][w] = c2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int u = 1; u < (int)(blockDim.x >> 5); u++) {
      c0 = cadd(c0, red[0][u]);
      c1 = cadd(c1, red[1][u]);
      c2 = cadd(c2, red[2][u]);
    }
    // rh x (rh x C) = rh (rh.C) - C for the unit direction rh
    const double2 d = cadd(cadd(cscale(c0, r0), cscale(c1, r1)), cscale(c2, r2));
    const double2 pref = make_double2(0, k * eta0 * DMB_INV_FOUR_PI);
    const double2 v0 = cmul(pref, csub(cscale(d, r0), c0));
    const double2 v1 = cmul(pref, csub(cscale(d, r1), c1));
    const double2 v2 = cmul(pref, csub(cscale(d, r2), c2));
    E[3 * r] = v0;
    E[3 * r + 1] = v1;
    E[3 * r + 2] = v2;
    const double e0 = E0s[r];
    sigma[r] = 4.0 * 3.14159265358979323846 * (cabs2(v0) + cabs2(v1) + cabs2(v2)) / (e0 * e0);
  }
}

// C (M x R col-major) = A (M x K row-major) B (K x R col-major)
__global__ void __launch_bounds__(256) k_gemm_rc(int64_t M, int64_t K, int64_t R, const double2 *__restrict__ A,
                                                 const double2 *__restrict__ B, double2 *__restrict__ C) {
  __shared__ double2 As[16][65];
  __shared__ double2 Bs[16][65];
  int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  int64_t m0 = (int64_t)blockIdx.x * 64, r0 = (int64_t)blockIdx.y * 64;
  double2 acc[4][4];
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) acc[i][j] = make_double2(0, 0);
  for (int64_t k0 = 0; k0 < K; k0 += 16) {
    for (int e = threadIdx.x; e < 16 * 64; e += 256) {
      int kk = e & 15, mm = e >> 4;
      int64_t m = m0 + mm, kx = k0 + kk, r = r0 + mm;
      As[kk][mm] = (m < M && kx < K) ? A[m * K + kx] : make_double2(0, 0);
      Bs[kk][mm] = (r < R && kx < K) ? B[r * K + kx] : make_double2(0, 0);
    }
    __syncthreads();
    for (int kk = 0; kk < 16; kk++)
      for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) acc[i][j] = cadd(acc[i][j], cmul(As[kk][ty + 16 * i], Bs[kk][tx + 16 * j]));
    __syncthreads();
  }
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      int64_t m = m0 + ty + 16 * i, r = r0 + tx + 16 * j;
      if (m < M && r < R) C[r * M + m] = acc[i][j];
    }
}

// ---------------------------------------------------------------------------
// matrix-free operator
// ---------------------------------------------------------------------------
__global__ void k_scatter_slots(int64_t N, const int *__restrict__ rslot, const double2 *__restrict__ x,
                                double2 *__restrict__ Xs) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= N) return;
  Xs[rslot[2 * m]] = x[m];
  Xs[rslot[2 * m + 1]] = x[m];
}

__device__ __forceinline__ bool tri_adjacent2(const int *__restrict__ off, const int *__restrict__ nb, int ta, int tb) {
  for (int i = off[ta]; i < off[ta + 1]; i++)
    if (nb[i] == tb) return true;
  return false;
}

// Ys[3ta+i] = sum_{tb far from ta} sum_j block(ta,tb)[i][j] Xs[3tb+j]
__global__ void __launch_bounds__(256) k_mf_far(int nt, int nq, const TriCache *__restrict__ tc,
                                                const int *__restrict__ aoff, const int *__restrict__ anb,
                                                double k, double inv_k2, const double2 *__restrict__ Xs,
                                                double2 *__restrict__ Ys) {
  __shared__ double2 red[8][3];
  int ta = blockIdx.x;
  const TriCache &A = tc[ta];
  double2 y[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
  for (int tb = threadIdx.x; tb < nt; tb += blockDim.x) {
    if (tb == ta || tri_adjacent2(aoff, anb, ta, tb)) continue;
    const TriCache &B = tc[tb];
    double2 xs[3];
    bool any = false;
    for (int j = 0; j < 3; j++) {
      xs[j] = B.rwg[j] >= 0 ? Xs[3 * tb + j] : make_double2(0, 0);
      any |= B.rwg[j] >= 0;
    }
    if (!any) continue;
    double m0r = 0, m0i = 0, mar[3] = {0, 0, 0}, mai[3] = {0, 0, 0}, mbr[3] = {0, 0, 0}, mbi[3] = {0, 0, 0},
           mabr = 0, mabi = 0;
    for (int b = 0; b < nq; b++)
      for (int a = 0; a < nq; a++) {
        double dx = A.qp[a][0] - B.qp[b][0], dy = A.qp[a][1] - B.qp[b][1], dz = A.qp[a][2] - B.qp[b][2];
        double R = sqrt(dx * dx + dy * dy + dz * dz);
        double sn, cs;
        sincos(k * R, &sn, &cs);
        double g = (DMB_INV_FOUR_PI / R) * (A.w2a[a] * B.w2a[b]);
        double gr = cs * g, gi = -sn * g;
        m0r += gr;
        m0i += gi;
        for (int d = 0; d < 3; d++) {
          mar[d] += gr * A.ql[a][d];
          mai[d] += gi * A.ql[a][d];
          mbr[d] += gr * B.ql[b][d];
          mbi[d] += gi * B.ql[b][d];
        }
        double dd = A.ql[a][0] * B.ql[b][0] + A.ql[a][1] * B.ql[b][1] + A.ql[a][2] * B.ql[b][2];
        mabr += gr * dd;
        mabi += gi * dd;
      }
    for (int i = 0; i < 3; i++) {
      if (A.rwg[i] < 0) continue;
      double mbpr = mbr[0] * A.pl[i][0] + mbr[1] * A.pl[i][1] + mbr[2] * A.pl[i][2];
      double mbpi = mbi[0] * A.pl[i][0] + mbi[1] * A.pl[i][1] + mbi[2] * A.pl[i][2];
      for (int j = 0; j < 3; j++) {
        if (B.rwg[j] < 0) continue;
        double mapr = mar[0] * B.pl[j][0] + mar[1] * B.pl[j][1] + mar[2] * B.pl[j][2];
        double mapi = mai[0] * B.pl[j][0] + mai[1] * B.pl[j][1] + mai[2] * B.pl[j][2];
        double pp = A.pl[i][0] * B.pl[j][0] + A.pl[i][1] * B.pl[j][1] + A.pl[i][2] * B.pl[j][2];
        double ss = A.s[i] * B.s[j], sc = A.dv[i] * B.dv[j] * inv_k2;
        double2 v = make_double2(ss * (mabr - mapr - mbpr + pp * m0r) - sc * m0r,
                                 ss * (mabi - mapi - mbpi + pp * m0i) - sc * m0i);
        y[i] = cadd(y[i], cmul(v, xs[j]));
      }
    }
  }
  for (int i = 0; i < 3; i++) {
    double2 v = warp_sum2(y[i]);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32][i] = v;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double2 s = make_double2(0, 0);
    for (int w = 0; w < 8; w++) s = cadd(s, red[w][threadIdx.x]);
    Ys[3 * ta + threadIdx.x] = s;
  }
}

__global__ void k_mf_gather(int64_t N, const int *__restrict__ rslot, const double2 *__restrict__ Ys,
                            double2 *__restrict__ y) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= N) return;
  y[m] = cadd(Ys[rslot[2 * m]], Ys[rslot[2 * m + 1]]);
}

// value of each near entry: its records summed in order (once per prepared
// operator)
__global__ void k_near_entry_sum(int64_t nent, const int64_t *__restrict__ off, const double2 *__restrict__ vals,
                                 double2 *__restrict__ esum) {
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nent) return;
  double2 v = make_double2(0, 0);
  for (int64_t r = off[e]; r < off[e + 1]; r++) v = cadd(v, vals[r]);
  esum[e] = v;
}

// near part per row, in the row's fixed entry order: y[m] += sum v_e x[other]
// (one thread per row, no atomics: repeated products are bitwise equal)
__global__ void k_mf_near_rows(int64_t N, const int64_t *__restrict__ roff, const int *__restrict__ rent,
                               const int *__restrict__ rcol, const double2 *__restrict__ esum,
                               const double2 *__restrict__ x, double2 *__restrict__ y) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= N) return;
  double2 acc = make_double2(0, 0);
  for (int64_t q = roff[m]; q < roff[m + 1]; q++) acc = cadd(acc, cmul(esum[rent[q]], x[rcol[q]]));
  y[m] = cadd(y[m], acc);
}

__global__ void k_times_minus_i_w(int64_t N, double w, double2 *__restrict__ y) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= N) return;
  double2 v = y[m];
  y[m] = make_double2(w * v.y, -w * v.x);
}

}  // namespace

namespace dmb {

void near_values(dmb_ctx *c, double k, double inv_k2);

void rhs_plane_waves_dev(dmb_ctx *c, const double *kvecs, const double *E0s, const double *pols, int64_t R,
                         int quad_order, double *V_dev) {
  double t0 = now_ms();
  rhs_plane_waves_async(c, kvecs, E0s, pols, R, quad_order, V_dev);
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  c->tm.rhs_ms = now_ms() - t0;
}

// the same without the final host synchronisation (the staging copies of the
// incidence data have completed when it returns: they come from pageable
// host memory)
void rhs_plane_waves_async(dmb_ctx *c, const double *kvecs, const double *E0s, const double *pols, int64_t R,
                           int quad_order, double *V_dev) {
  ensure_cache(c, quad_order);
  c->d_small.ensure(std::max<size_t>(65536, 64 + sizeof(double) * 7 * R));
  double *dk = (double *)((char *)c->d_small.p + 64), *de = dk + 3 * R, *dp = de + R;
  DMB_CUDA(cudaMemcpyAsync(dk, kvecs, 24 * R, cudaMemcpyHostToDevice, c->stream));
  DMB_CUDA(cudaMemcpyAsync(de, E0s, 8 * R, cudaMemcpyHostToDevice, c->stream));
  DMB_CUDA(cudaMemcpyAsync(dp, pols, 24 * R, cudaMemcpyHostToDevice, c->stream));
  DMB_LAUNCH(c, k_plane_wave, blocks_for(c->n * R, 128), 128, 0, c->n, R, c->d_tcache.as<TriCache>(),
             c->d_rwg_slot.as<int>(), c->nq, c->d_wq.as<double>(), dk, de, dp, (double2 *)V_dev);
}

void farfield_dev(dmb_ctx *c, const double *rhat, int64_t NO, double k, double eta0, int quad_order,
                  const double *I_dev, int64_t nrhs, double *E_dev) {
  ensure_cache(c, quad_order);
  const int64_t N = c->n;
  DevBuf dr, G;
  dr.ensure(24 * NO);
  G.ensure(sizeof(double2) * 3 * NO * N);
  DMB_CUDA(cudaMemcpyAsync(dr.p, rhat, 24 * NO, cudaMemcpyHostToDevice, c->stream));
  dim3 g(blocks_for(N, 128), (unsigned)NO);
  DMB_LAUNCH(c, k_radiation, g, 128, 0, N, NO, c->d_tcache.as<TriCache>(), c->d_rwg_slot.as<int>(), c->nq,
             c->d_wq.as<double>(), dr.as<double>(), k, eta0, G.as<double2>());
  dim3 g2(blocks_for(3 * NO, 64), blocks_for(nrhs, 64));
  DMB_LAUNCH(c, k_gemm_rc, g2, 256, 0, 3 * NO, N, nrhs, G.as<double2>(), (const double2 *)I_dev,
             (double2 *)E_dev);
  DMB_CUDA(cudaStreamSynchronize(c->stream));
}

void rhs_dipoles_dev(dmb_ctx *c, int64_t R, const double *pos, const double *moments, const int *magnetic,
                     const double *freqs, int quad_order, double *V_dev) {
  double t0 = now_ms();
  ensure_cache(c, quad_order);
  DevBuf bp, bm, bt, bf;
  bp.ensure(24 * R);
  bm.ensure(48 * R);
  bt.ensure(4 * R);
  bf.ensure(8 * R);
  DMB_CUDA(cudaMemcpyAsync(bp.p, pos, 24 * R, cudaMemcpyHostToDevice, c->stream));
  DMB_CUDA(cudaMemcpyAsync(bm.p, moments, 48 * R, cudaMemcpyHostToDevice, c->stream));
  DMB_CUDA(cudaMemcpyAsync(bt.p, magnetic, 4 * R, cudaMemcpyHostToDevice, c->stream));
  DMB_CUDA(cudaMemcpyAsync(bf.p, freqs, 8 * R, cudaMemcpyHostToDevice, c->stream));
  DMB_LAUNCH(c, k_dipole_rhs, blocks_for(c->n * R, 128), 128, 0, c->n, R, c->d_tcache.as<TriCache>(),
             c->d_rwg_slot.as<int>(), c->nq, c->d_wq.as<double>(), bp.as<double>(), bm.as<double>(), bt.as<int>(),
             bf.as<double>(), (double2 *)V_dev);
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  c->tm.rhs_ms = now_ms() - t0;
}

void rhs_pattern_dev(dmb_ctx *c, int nth, const double *theta, int nph, const double *phi, const double *Ft,
                     const double *Fp, double freq, const double *pc, int conj_conv, int quad_order, double *V_dev) {
  double t0 = now_ms();
  ensure_cache(c, quad_order);
  DevBuf bth, bph, bft, bfp;
  const size_t nf = (size_t)nth * nph;
  bth.ensure(8 * nth);
  bph.ensure(8 * nph);
  bft.ensure(16 * nf);
  bfp.ensure(16 * nf);
  DMB_CUDA(cudaMemcpyAsync(bth.p, theta, 8 * nth, cudaMemcpyHostToDevice, c->stream));
  DMB_CUDA(cudaMemcpyAsync(bph.p, phi, 8 * nph, cudaMemcpyHostToDevice, c->stream));
  DMB_CUDA(cudaMemcpyAsync(bft.p, Ft, 16 * nf, cudaMemcpyHostToDevice, c->stream));
  DMB_CUDA(cudaMemcpyAsync(bfp.p, Fp, 16 * nf, cudaMemcpyHostToDevice, c->stream));
  PatternDev P;
  P.nth = nth;
  P.nph = nph;
  P.th = bth.as<double>();
  P.ph = bph.as<double>();
  P.Ft = (const double2 *)bft.p;
  P.Fp = (const double2 *)bfp.p;
  P.k = 2.0 * 3.14159265358979323846 * freq / 299792458.0;
  for (int a = 0; a < 3; a++) P.pc[a] = pc[a];
  P.conj = conj_conv;
  DMB_LAUNCH(c, k_pattern_rhs, blocks_for(c->n, 128), 128, 0, c->n, c->d_tcache.as<TriCache>(),
             c->d_rwg_slot.as<int>(), c->nq, c->d_wq.as<double>(), P, (double2 *)V_dev);
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  c->tm.rhs_ms = now_ms() - t0;
}

// monostatic fields of R resident solutions; kv / E0s are the device copies
// that rhs_plane_waves_dev staged in d_small
void monostatic_dev(dmb_ctx *c, int64_t R, double k, double eta0, int quad_order, const double *I_dev,
                    double *E_dev, double *sigma_dev) {
  ensure_cache(c, quad_order);
  const double *dk = (const double *)((const char *)c->d_small.p + 64), *de = dk + 3 * R;
  DMB_LAUNCH(c, k_monostatic, (unsigned)R, 256, 0, c->n, c->d_tcache.as<TriCache>(), c->d_rwg_slot.as<int>(),
             c->nq, c->d_wq.as<double>(), dk, de, k, eta0, (const double2 *)I_dev, (double2 *)E_dev, sigma_dev);
}

void prepare_operator(dmb_ctx *c, double k, double eta0, int quad_order) {
  DMB_REQUIRE(std::isfinite(k) && k != 0.0, DMB_ERR_ARGUMENT, "EFIE wavenumber must be finite and nonzero");
  DMB_REQUIRE(std::isfinite(eta0) && eta0 != 0.0, DMB_ERR_ARGUMENT, "EFIE eta0 must be finite and nonzero");
  ensure_cache(c, quad_order);
  c->k = k;
  c->eta0 = eta0;
  near_values(c, k, 1.0 / (k * k));
}

void matvec_free_dev(dmb_ctx *c, const double *x, double *y) {
  DMB_REQUIRE(c->cache_valid && c->k != 0.0, DMB_ERR_STATE, "operator not prepared");
  const int64_t N = c->n, nt = c->nt;
  DevBuf xs, ys;
  xs.ensure(sizeof(double2) * 3 * nt);
  ys.ensure(sizeof(double2) * 3 * nt);
  DMB_CUDA(cudaMemsetAsync(xs.p, 0, sizeof(double2) * 3 * nt, c->stream));
  DMB_LAUNCH(c, k_scatter_slots, blocks_for(N, 256), 256, 0, N, c->d_rwg_slot.as<int>(), (const double2 *)x,
             xs.as<double2>());
  DMB_LAUNCH(c, k_mf_far, (unsigned)nt, 256, 0, (int)nt, c->nq, c->d_tcache.as<TriCache>(),
             c->d_adj_off.as<int>(), c->d_adj_nb.as<int>(), c->k, 1.0 / (c->k * c->k), xs.as<double2>(),
             ys.as<double2>());
  DMB_LAUNCH(c, k_mf_gather, blocks_for(N, 256), 256, 0, N, c->d_rwg_slot.as<int>(), ys.as<double2>(),
             (double2 *)y);
  if (c->n_near_entry > 0) {
    DMB_LAUNCH(c, k_near_entry_sum, blocks_for(c->n_near_entry, 256), 256, 0, c->n_near_entry,
               c->d_near_entry_off.as<int64_t>(), c->d_near_val.as<double2>(), c->d_near_entry_sum.as<double2>());
    DMB_LAUNCH(c, k_mf_near_rows, blocks_for(N, 256), 256, 0, N, c->d_near_row_off.as<int64_t>(),
               c->d_near_row_ent.as<int>(), c->d_near_row_col.as<int>(), c->d_near_entry_sum.as<double2>(),
               (const double2 *)x, (double2 *)y);
  }
  DMB_LAUNCH(c, k_times_minus_i_w, blocks_for(N, 256), 256, 0, N, c->k * c->eta0, (double2 *)y);
  DMB_CUDA(cudaStreamSynchronize(c->stream));
}

}  // namespace dmb

// ---------------------------------------------------------------------------
// Matrix-free product that allocates nothing.
//
// Some callers cannot allocate device memory in the middle of a run: codes
// whose device memory is owned by an external pool (a framework allocator that
// must see every byte), or fixed-budget solvers that forbid allocation after
// set-up.  dmb_matvec_free_noalloc serves them: the caller passes device
// input/output vectors, and the slot-space scratch of the product lives in the
// file-scope array below instead of per-call cudaMalloc buffers.
// ---------------------------------------------------------------------------
namespace {

constexpr int64_t kNoAllocMaxTriangles = 32768;
// slot-space input (first half) and output (second half): 2 x 3 x max triangles
// complex128 = 3 MiB, held by every GPU that loads the library until exit.
static __device__ __align__(256) double2 g_mf_noalloc_scratch[2 * 3 * kNoAllocMaxTriangles];

// Host code must not use g_mf_noalloc_scratch directly (its host-side name is a
// stand-in, not a device address).  The address is looked up on every call,
// with the context's device current: cudaGetSymbolAddress allocates nothing,
// and a fresh lookup stays right if the device's context was reset and the
// module reloaded elsewhere since an earlier call.
double2 *noalloc_scratch() {
  void *p = nullptr;
  DMB_CUDA(cudaGetSymbolAddress(&p, g_mf_noalloc_scratch));
  return static_cast<double2 *>(p);
}

}  // namespace

extern "C" dmb_status dmb_matvec_free_noalloc(dmb_ctx *c, const double *x_dev, double *y_dev) {
  if (!c) return DMB_ERR_ARGUMENT;
  std::lock_guard<std::mutex> lk(c->mu);
  try {
    DMB_CUDA(cudaSetDevice(c->device));
    DMB_REQUIRE(x_dev && y_dev, DMB_ERR_ARGUMENT, "x and y must be device pointers");
    DMB_REQUIRE(c->cache_valid && c->k != 0.0, DMB_ERR_STATE,
                "operator not prepared: call dmb_prepare_operator first");
    DMB_REQUIRE(c->nt <= kNoAllocMaxTriangles, DMB_ERR_BUDGET,
                "dmb_matvec_free_noalloc supports at most " + std::to_string(kNoAllocMaxTriangles) +
                    " triangles, mesh has " + std::to_string(c->nt));
    const int64_t N = c->n, nt = c->nt;
    double2 *xs = noalloc_scratch();
    double2 *ys = xs + 3 * kNoAllocMaxTriangles;
    // slots without a basis function are never read, but the input half is
    // cleared so no value of an earlier call can leak into this one
    DMB_CUDA(cudaMemsetAsync(xs, 0, sizeof(double2) * 3 * nt, c->stream));
    DMB_LAUNCH(c, k_scatter_slots, blocks_for(N, 256), 256, 0, N, c->d_rwg_slot.as<int>(),
               (const double2 *)x_dev, xs);
    DMB_LAUNCH(c, k_mf_far, (unsigned)nt, 256, 0, (int)nt, c->nq, c->d_tcache.as<TriCache>(),
               c->d_adj_off.as<int>(), c->d_adj_nb.as<int>(), c->k, 1.0 / (c->k * c->k), xs, ys);
    DMB_LAUNCH(c, k_mf_gather, blocks_for(N, 256), 256, 0, N, c->d_rwg_slot.as<int>(), ys, (double2 *)y_dev);
    if (c->n_near_entry > 0) {
      DMB_LAUNCH(c, k_near_entry_sum, blocks_for(c->n_near_entry, 256), 256, 0, c->n_near_entry,
                 c->d_near_entry_off.as<int64_t>(), c->d_near_val.as<double2>(), c->d_near_entry_sum.as<double2>());
      DMB_LAUNCH(c, k_mf_near_rows, blocks_for(N, 256), 256, 0, N, c->d_near_row_off.as<int64_t>(),
                 c->d_near_row_ent.as<int>(), c->d_near_row_col.as<int>(), c->d_near_entry_sum.as<double2>(),
                 (const double2 *)x_dev, (double2 *)y_dev);
    }
    DMB_LAUNCH(c, k_times_minus_i_w, blocks_for(N, 256), 256, 0, N, c->k * c->eta0, (double2 *)y_dev);
    DMB_CUDA(cudaStreamSynchronize(c->stream));
    c->err.clear();
    return DMB_OK;
  } catch (const DmbError &e) {
    c->err = e.msg;
    return e.code;
  }
}
