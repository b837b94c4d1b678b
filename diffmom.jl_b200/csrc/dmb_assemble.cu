// dmb_assemble.cu -- cache precompute and impedance-matrix assembly.
//
// Reference path: assemble_Z_efie (src/assembly/EFIE.jl:699-753) evaluates
// every RWG pair (m <= n) as a sum over its 2x2 triangle pairs
// (_efie_entry, EFIE.jl:439-512).  Here:
//
//   far pairs   (not self, not edge-adjacent): dmb_fartile.cu, one CTA per
//               tile of RWG pairs, triangle panels staged in shared memory,
//               Z entries written directly (the four triangle pairs of an
//               entry summed in a fixed order).
//   near pairs  self (EFIE.jl:534-606) and edge-adjacent (EFIE.jl:611-684)
//               terms are evaluated per (pair, test slot, source slot) record
//               with the reference's canonical rule (the lower RWG index is
//               the test function: outer 7-point quadrature on its triangle,
//               analytic 1/R on the source triangle), then summed per entry
//               in a fixed order and added to Z -- no atomics, deterministic.
//
// Z is complex symmetric, so its row-major and column-major layouts coincide.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include "dmb_device.cuh"
#include "dmb_internal.h"

namespace {

// ---------------------------------------------------------------------------
// quadrature rules (Quadrature.jl:17-54)
// ---------------------------------------------------------------------------
int quad_rule(int order, double *x1, double *x2, double *w) {
  if (order == 1) {
    x1[0] = 1.0 / 3; x2[0] = 1.0 / 3; w[0] = 0.5;
    return 1;
  }
  if (order == 3) {
    x1[0] = 1.0 / 6; x2[0] = 1.0 / 6;
    x1[1] = 2.0 / 3; x2[1] = 1.0 / 6;
    x1[2] = 1.0 / 6; x2[2] = 2.0 / 3;
    w[0] = w[1] = w[2] = 1.0 / 6;
    return 3;
  }
  if (order == 4) {
    x1[0] = 1.0 / 3; x2[0] = 1.0 / 3;
    x1[1] = 0.6; x2[1] = 0.2;
    x1[2] = 0.2; x2[2] = 0.6;
    x1[3] = 0.2; x2[3] = 0.2;
    w[0] = -27.0 / 96; w[1] = w[2] = w[3] = 25.0 / 96;
    return 4;
  }
  if (order == 7) {
    const double a1 = 0.059715871789770, b1 = 0.470142064105115;
    const double a2 = 0.797426985353087, b2 = 0.101286507323456;
    const double px[7] = {1.0 / 3, b1, a1, b1, b2, a2, b2};
    const double py[7] = {1.0 / 3, b1, b1, a1, b2, b2, a2};
    for (int i = 0; i < 7; i++) { x1[i] = px[i]; x2[i] = py[i]; }
    w[0] = 0.1125;
    w[1] = w[2] = w[3] = 0.0661970763942530;
    w[4] = w[5] = w[6] = 0.0629695902724135;
    return 7;
  }
  return -1;
}

struct QuadConst {
  double x1[7], x2[7], h1[7], h2[7], w[7], wh[7];
  int nq;
};

// ---------------------------------------------------------------------------
// device geometry helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dd_two_sum(double a, double b, double &s, double &e) {
  s = a + b;
  double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

// w1*a + x1*b + x2*c with w1 = 1 - x1 - x2 kept in double-double; replaces
// the BigFloat branch of _triangle_affine_component (Quadrature.jl:57-74).
__device__ double affine_exact(double a, double b, double c, double x1, double x2) {
  double s1, e1, s2, e2;
  dd_two_sum(1.0, -x1, s1, e1);
  dd_two_sum(s1, -x2, s2, e2);
  double wl = e1 + e2;
  double p1 = s2 * a, q1 = fma(s2, a, -p1) + wl * a;
  double p2 = x1 * b, q2 = fma(x1, b, -p2);
  double p3 = x2 * c, q3 = fma(x2, c, -p3);
  double s, e, t, f;
  dd_two_sum(p1, p2, s, e);
  dd_two_sum(s, p3, t, f);
  return t + (e + f + q1 + q2 + q3);
}

// Quadrature.jl:76-113 _triangle_affine_component (muladd with a
// cancellation test that routes to the exact evaluation).
__device__ double affine_component(double a, double b, double c, double x1, double x2) {
  double w1 = 1.0 - x1 - x2;
  double pa = __dmul_rn(w1, a), pb = __dmul_rn(x1, b), pc = __dmul_rn(x2, c);
  if (!isfinite(pa) || !isfinite(pb) || !isfinite(pc)) return affine_exact(a, b, c, x1, x2);
  if ((pa == 0.0 && w1 != 0.0 && a != 0.0) || (pb == 0.0 && x1 != 0.0 && b != 0.0) ||
      (pc == 0.0 && x2 != 0.0 && c != 0.0))
    return affine_exact(a, b, c, x1, x2);
  double asum = fabs(pa) + fabs(pb) + fabs(pc);
  if (!isfinite(asum)) return affine_exact(a, b, c, x1, x2);
  double value = fma(w1, a, fma(x1, b, pc));
  if (!isfinite(value) || (asum != 0.0 && fabs(value) <= 64 * 2.220446049250313e-16 * asum) ||
      (value != 0.0 && fabs(value) < 2.2250738585072014e-308))
    return affine_exact(a, b, c, x1, x2);
  return value;
}

// Mesh.jl:2966-3080: power-of-two scaled cross product area.
__device__ double tri_area(const double *v1, const double *v2, const double *v3) {
  double e1x = v2[0] - v1[0], e1y = v2[1] - v1[1], e1z = v2[2] - v1[2];
  double e2x = v3[0] - v1[0], e2y = v3[1] - v1[1], e2z = v3[2] - v1[2];
  double s1 = fmax(fabs(e1x), fmax(fabs(e1y), fabs(e1z)));
  double s2 = fmax(fabs(e2x), fmax(fabs(e2y), fabs(e2z)));
  if (!(s1 > 0 && s2 > 0)) return 0.0;
  int x1, x2;
  frexp(s1, &x1);
  frexp(s2, &x2);
  double a1 = ldexp(e1x, -x1), a2 = ldexp(e1y, -x1), a3 = ldexp(e1z, -x1);
  double b1 = ldexp(e2x, -x2), b2 = ldexp(e2y, -x2), b3 = ldexp(e2z, -x2);
  double cx = __dsub_rn(__dmul_rn(a2, b3), __dmul_rn(a3, b2));
  double cy = __dsub_rn(__dmul_rn(a3, b1), __dmul_rn(a1, b3));
  double cz = __dsub_rn(__dmul_rn(a1, b2), __dmul_rn(a2, b1));
  double cn = hypot(hypot(cx, cy), cz);
  if (cn == 0.0) return 0.0;
  int xn;
  double fn = frexp(cn, &xn);
  return ldexp(0.5 * fn, xn + x1 + x2);
}

__device__ double mean3(double a, double b, double c) {
  double s12, e12, s123, e3, cl, ce, sl, se;
  dd_two_sum(a, b, s12, e12);
  dd_two_sum(s12, c, s123, e3);
  dd_two_sum(e12, e3, cl, ce);
  dd_two_sum(s123, cl, sl, se);
  return (sl + (se + ce)) / 3.0;
}

// K1: per-triangle cache (EFIE.jl:355-397).  slot_rwg/slot_side come from the
// host topology pass; RWG length/areas/opposite vertices from the upload.
__global__ void k_tri_cache(int nt, const double *__restrict__ xyz, const int *__restrict__ tri,
                            const int *__restrict__ slot_rwg, const int *__restrict__ slot_side,
                            const double *__restrict__ len, const double *__restrict__ ap,
                            const double *__restrict__ am, const int *__restrict__ vpo,
                            const int *__restrict__ vmo, QuadConst qc, TriCache *__restrict__ out) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  TriCache c;
  for (int a = 0; a < 3; a++)
    for (int d = 0; d < 3; d++) c.v[a][d] = xyz[3 * tri[3 * t + a] + d];
  c.area = tri_area(c.v[0], c.v[1], c.v[2]);
  for (int d = 0; d < 3; d++) c.cen[d] = mean3(c.v[0][d], c.v[1][d], c.v[2][d]);
  for (int q = 0; q < 7; q++) {
    for (int d = 0; d < 3; d++) {
      double x = 0.0, xh;
      if (q < qc.nq) x = affine_component(c.v[0][d], c.v[1][d], c.v[2][d], qc.x1[q], qc.x2[q]);
      xh = affine_component(c.v[0][d], c.v[1][d], c.v[2][d], qc.h1[q], qc.h2[q]);
      c.qp[q][d] = x;
      c.qph[q][d] = xh;
      c.ql[q][d] = x - c.cen[d];
    }
    c.w2a[q] = q < qc.nq ? qc.w[q] * (2.0 * c.area) : 0.0;
    c.w2ah[q] = qc.wh[q] * (2.0 * c.area);
  }
  for (int i = 0; i < 3; i++) {
    int n = slot_rwg[3 * t + i];
    c.rwg[i] = n;
    c.side[i] = slot_side[3 * t + i];
    if (n < 0) {
      c.s[i] = 0.0;
      c.dv[i] = 0.0;
      for (int d = 0; d < 3; d++) c.p[i][d] = c.pl[i][d] = 0.0;
      continue;
    }
    // RWG.jl:763-807: f = (len/(2A)) (r - r_opp) on T+, (len/(2A)) (r_opp - r)
    // on T-; div = +len/A+, -len/A-.
    bool plus = c.side[i] == 0;
    double A = plus ? ap[n] : am[n];
    double sr = len[n] / (2.0 * A);
    c.s[i] = plus ? sr : -sr;
    c.dv[i] = plus ? 1.0 * (len[n] / A) : -1.0 * (len[n] / A);
    int ov = plus ? vpo[n] : vmo[n];
    for (int d = 0; d < 3; d++) {
      c.p[i][d] = xyz[3 * ov + d];
      c.pl[i][d] = c.p[i][d] - c.cen[d];
    }
  }
  out[t] = c;
}

// centres of RWG functions (NearFieldPreconditioner.jl:247-257)
__global__ void k_rwg_centers(int n, const TriCache *__restrict__ tc, const int *__restrict__ tp,
                              const int *__restrict__ tm, double *__restrict__ centers) {
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  for (int d = 0; d < 3; d++) {
    double a = tc[tp[m]].cen[d], b = tc[tm[m]].cen[d];
    double lo = fmin(a, b), hi = fmax(a, b);
    if (a == b) { lo = a; hi = b; }
    double mid = (signbit(lo) == signbit(hi)) ? lo + (hi - lo) / 2 : (lo + hi) / 2;
    centers[3 * m + d] = mid;
  }
}

// ---------------------------------------------------------------------------
// near-singular terms (device restatement of EFIE.jl:534-684 and
// SingularIntegrals.jl:146-203)
// ---------------------------------------------------------------------------
__device__ double analytic_1overR(const double P[3], const double V1[3], const double V2[3],
                                  const double V3[3]) {
  double e1[3] = {V2[0] - V1[0], V2[1] - V1[1], V2[2] - V1[2]};
  double e2[3] = {V3[0] - V1[0], V3[1] - V1[1], V3[2] - V1[2]};
  double nT[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                  e1[0] * e2[1] - e1[1] * e2[0]};
  double nn = sqrt(nT[0] * nT[0] + nT[1] * nT[1] + nT[2] * nT[2]);
  if (nn == 0.0) return 0.0;
  nT[0] /= nn; nT[1] /= nn; nT[2] /= nn;
  double h = (P[0] - V1[0]) * nT[0] + (P[1] - V1[1]) * nT[1] + (P[2] - V1[2]) * nT[2];
  double ah = fabs(h);
  double xi[3] = {P[0] - h * nT[0], P[1] - h * nT[1], P[2] - h * nT[2]};
  const double *As[3] = {V1, V2, V3};
  const double *Bs[3] = {V2, V3, V1};
  double log_sum = 0.0, atan_sum = 0.0;
  for (int e = 0; e < 3; e++) {
    const double *A = As[e], *B = Bs[e];
    double ev[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]};
    double el = sqrt(ev[0] * ev[0] + ev[1] * ev[1] + ev[2] * ev[2]);
    if (el == 0.0) continue;
    double lh[3] = {ev[0] / el, ev[1] / el, ev[2] / el};
    double nh[3] = {lh[1] * nT[2] - lh[2] * nT[1], lh[2] * nT[0] - lh[0] * nT[2],
                    lh[0] * nT[1] - lh[1] * nT[0]};
    double ax[3] = {A[0] - xi[0], A[1] - xi[1], A[2] - xi[2]};
    double bx[3] = {B[0] - xi[0], B[1] - xi[1], B[2] - xi[2]};
    double d = ax[0] * nh[0] + ax[1] * nh[1] + ax[2] * nh[2];
    double sm = ax[0] * lh[0] + ax[1] * lh[1] + ax[2] * lh[2];
    double sp = bx[0] * lh[0] + bx[1] * lh[1] + bx[2] * lh[2];
    double pa[3] = {P[0] - A[0], P[1] - A[1], P[2] - A[2]};
    double pb[3] = {P[0] - B[0], P[1] - B[1], P[2] - B[2]};
    double Rm = sqrt(pa[0] * pa[0] + pa[1] * pa[1] + pa[2] * pa[2]);
    double Rp = sqrt(pb[0] * pb[0] + pb[1] * pb[1] + pb[2] * pb[2]);
    double R0sq = d * d + h * h;
    if (d != 0.0) {
      double den = sm + Rm, num = sp + Rp;
      if (den > 0.0 && num > 0.0) log_sum += d * log(num / den);
    }
    if (ah != 0.0 && d != 0.0) {
      double apl = atan(d * sp / (R0sq + ah * Rp));
      double ami = atan(d * sm / (R0sq + ah * Rm));
      atan_sum += apl - ami;
    }
  }
  return log_sum - ah * atan_sum;
}

// Greens.jl:189-201 compensated exprel series, 18 terms
__device__ double2 green_exprel(double2 z) {
  double2 term = make_double2(1.0, 0.0), total = term, corr = make_double2(0.0, 0.0);
  for (int order = 1; order <= 18; order++) {
    double2 zs = make_double2(z.x / (order + 1), z.y / (order + 1));
    term = cmul(term, zs);
    double2 ct = csub(term, corr);
    double2 upd = cadd(total, ct);
    corr = csub(csub(upd, total), ct);
    total = upd;
  }
  return total;
}

// Greens.jl:381-400 _greens_smooth_unchecked: (exp(-ikR)-1)/(4 pi R)
__device__ double2 greens_smooth(const double r[3], const double rp[3], double k) {
  double dx = r[0] - rp[0], dy = r[1] - rp[1], dz = r[2] - rp[2];
  double R = hypot(hypot(dx, dy), dz);
  double2 q = make_double2(0.0, -k);
  if (R == 0.0) return cscale(q, DMB_INV_FOUR_PI);
  double2 z = make_double2(0.0, -k * R);
  if (hypot(z.x, z.y) <= 0.5) return cmul(cscale(q, DMB_INV_FOUR_PI), green_exprel(z));
  double sh = sin(0.5 * z.y);
  double2 em1 = make_double2(0.0 - 2.0 * (sh * sh), sin(z.y));
  return cscale(em1, DMB_INV_FOUR_PI / R);
}

__device__ __forceinline__ void fval(const TriCache &T, int slot, const double r[3], double f[3]) {
  double s = T.s[slot];
  f[0] = s * (r[0] - T.p[slot][0]);
  f[1] = s * (r[1] - T.p[slot][1]);
  f[2] = s * (r[2] - T.p[slot][2]);
}
__device__ __forceinline__ double dot3(const double a[3], const double b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// one near record: self (ta == tb) or edge-adjacent (ta outer, tb analytic)
__device__ double2 near_value(const NearRec rc, const TriCache *__restrict__ tc, int nq,
                              const double *__restrict__ wq_std, const double *__restrict__ wq_hi, double k,
                              double inv_k2) {
  const TriCache &A = tc[rc.ta];
  const TriCache &B = tc[rc.tb];
  double dvm = A.dv[rc.ia], dvn = B.dv[rc.ib];
  double dvmn = dvm * dvn * inv_k2;
  double inv4pi = DMB_INV_FOUR_PI;
  double vr = 0, vi = 0;
  if (rc.ta == rc.tb) {
    // _self_cell_cached (EFIE.jl:534-606)
    double Am = A.area;
    double2 vs = make_double2(0, 0);
    for (int a = 0; a < 7; a++) {
      double fm[3];
      fval(A, rc.ia, A.qph[a], fm);
      for (int b = 0; b < 7; b++) {
        double fn[3];
        fval(A, rc.ib, A.qph[b], fn);
        double2 Gs = greens_smooth(A.qph[a], A.qph[b], k);
        double fd = dot3(fm, fn);
        double2 vp = cscale(Gs, fd), sp = cscale(Gs, dvmn);
        double wt = wq_hi[a] * wq_hi[b] * (2 * Am) * (2 * Am);
        vs = cadd(vs, cscale(csub(vp, sp), wt));
      }
    }
    double vg = 0.0;
    for (int a = 0; a < 7; a++) {
      double fm[3], fna[3];
      fval(A, rc.ia, A.qph[a], fm);
      fval(A, rc.ib, A.qph[a], fna);
      double S = analytic_1overR(A.qph[a], A.v[0], A.v[1], A.v[2]);
      double inner = inv4pi * S;
      double scl = dvmn * inner;
      double lead = dot3(fm, fna) * inner;
      double rem = 0.0;
      for (int b = 0; b < 7; b++) {
        double dx = A.qph[a][0] - A.qph[b][0], dy = A.qph[a][1] - A.qph[b][1],
               dz = A.qph[a][2] - A.qph[b][2];
        double R = hypot(hypot(dx, dy), dz);
        if (R == 0.0) continue;
        double fn[3];
        fval(A, rc.ib, A.qph[b], fn);
        double df[3] = {fn[0] - fna[0], fn[1] - fna[1], fn[2] - fna[2]};
        rem += dot3(fm, df) * (inv4pi / R) * wq_hi[b] * (2 * Am);
      }
      double ow = wq_hi[a] * (2 * Am);
      vg += ((lead + rem) - scl) * ow;
    }
    vr = vs.x + vg;
    vi = vs.y;
  } else {
    // _adjacent_cell_cached (EFIE.jl:611-684): smooth part on the standard
    // rule, singular part with outer 7-point rule on A, analytic on B.
    double Am = A.area, An = B.area;
    double2 vs = make_double2(0, 0);
    for (int a = 0; a < nq; a++) {
      double fm[3];
      fval(A, rc.ia, A.qp[a], fm);
      for (int b = 0; b < nq; b++) {
        double fn[3];
        fval(B, rc.ib, B.qp[b], fn);
        double2 Gs = greens_smooth(A.qp[a], B.qp[b], k);
        double2 vp = cscale(Gs, dot3(fm, fn)), sp = cscale(Gs, dvmn);
        double wt = wq_std[a] * wq_std[b] * (2 * Am) * (2 * An);
        vs = cadd(vs, cscale(csub(vp, sp), wt));
      }
    }
    double vg = 0.0;
    for (int a = 0; a < 7; a++) {
      double fm[3];
      fval(A, rc.ia, A.qph[a], fm);
      double S = analytic_1overR(A.qph[a], B.v[0], B.v[1], B.v[2]);
      double inner = inv4pi * S;
      double scl = dvmn * inner;
      double vsg = 0.0;
      for (int b = 0; b < 7; b++) {
        double dx = A.qph[a][0] - B.qph[b][0], dy = A.qph[a][1] - B.qph[b][1],
               dz = A.qph[a][2] - B.qph[b][2];
        double R = hypot(hypot(dx, dy), dz);
        if (R == 0.0) continue;
        double fn[3];
        fval(B, rc.ib, B.qph[b], fn);
        vsg += dot3(fm, fn) * (inv4pi / R) * wq_hi[b] * (2 * An);
      }
      double ow = wq_hi[a] * (2 * Am);
      vg += (vsg - scl) * ow;
    }
    vr = vs.x + vg;
    vi = vs.y;
  }
  return make_double2(vr, vi);
}

__global__ void k_near_values(int64_t nrec, const NearRec *__restrict__ recs,
                              const TriCache *__restrict__ tc, int nq, const double *__restrict__ wq_std,
                              const double *__restrict__ wq_hi, double k, double inv_k2,
                              double2 *__restrict__ vals) {
  int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrec) return;
  vals[r] = near_value(recs[r], tc, nq, wq_std, wq_hi, k, inv_k2);
}

// sum the records of each near entry in fixed order, add to Z[m][n], Z[n][m]
template <class ZC>
__device__ __forceinline__ void near_add_entry(int64_t e, const int2 *__restrict__ mn,
                                               const int64_t *__restrict__ off, const double2 *__restrict__ vals,
                                               double omega_mu0, int64_t N, ZC *__restrict__ Z) {
  double re = 0, im = 0;
  for (int64_t r = off[e]; r < off[e + 1]; r++) {
    re += vals[r].x;
    im += vals[r].y;
  }
  int2 p = mn[e];
  double2 add = make_double2(omega_mu0 * im, -omega_mu0 * re);
  ZC *a = Z + (int64_t)p.x * N + p.y;
  store_c(a, cadd(to_d2(*a), add));
  if (p.x != p.y) {
    ZC *b = Z + (int64_t)p.y * N + p.x;
    store_c(b, cadd(to_d2(*b), add));
  }
}

template <class ZC>
__global__ void k_near_add(int64_t nent, const int2 *__restrict__ mn, const int64_t *__restrict__ off,
                           const double2 *__restrict__ vals, double omega_mu0, int64_t N,
                           ZC *__restrict__ Z) {
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nent) return;
  near_add_entry(e, mn, off, vals, omega_mu0, N, Z);
}

// Near terms of many surfaces in one launch each (uneven surface batches):
// thread -> (surface, record / entry) through the jobs' prefix offsets.
struct NearJob {
  const NearRec *recs;
  const TriCache *tc;
  const double *wq;       // 7 standard + 7 high-order weights
  double2 *vals;
  const int2 *mn;
  const int64_t *eoff;
  void *Z;
  int64_t N, rec0, ent0;  // first record / entry of the surface in the batch
  double k, inv_k2, omega_mu0;
  int nq;
};

__device__ __forceinline__ int near_job_of(const NearJob *jobs, int njobs, int64_t g, bool entries) {
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if ((entries ? jobs[mid].ent0 : jobs[mid].rec0) <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void k_near_values_batched(const NearJob *__restrict__ jobs, int njobs, int64_t total) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total) return;
  const NearJob &jb = jobs[near_job_of(jobs, njobs, g, false)];
  const int64_t r = g - jb.rec0;
  jb.vals[r] = near_value(jb.recs[r], jb.tc, jb.nq, jb.wq, jb.wq + 7, jb.k, jb.inv_k2);
}

template <class ZC>
__global__ void k_near_add_batched(const NearJob *__restrict__ jobs, int njobs, int64_t total) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total) return;
  const NearJob &jb = jobs[near_job_of(jobs, njobs, g, true)];
  near_add_entry(g - jb.ent0, jb.mn, jb.eoff, jb.vals, jb.omega_mu0, jb.N, reinterpret_cast<ZC *>(jb.Z));
}

}  // namespace

namespace dmb {

double now_ms() {
  return std::chrono::duration<double, std::milli>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// Host topology: edge adjacency (EFIE.jl:140-231), basis slots per triangle,
// near-field records grouped by entry.  Integer bookkeeping, O(Nt log Nt).
void build_host_topology(dmb_ctx *c) {
  const int64_t nt = c->nt, N = c->n;
  // adjacency from sorted edge records
  std::vector<std::array<int32_t, 3>> rec;
  rec.reserve(3 * nt);
  for (int64_t t = 0; t < nt; t++)
    for (int e = 0; e < 3; e++) {
      int32_t a = c->h_tri[3 * t + e], b = c->h_tri[3 * t + (e + 1) % 3];
      rec.push_back({std::min(a, b), std::max(a, b), (int32_t)t});
    }
  std::sort(rec.begin(), rec.end());
  std::vector<std::pair<int32_t, int32_t>> pairs;
  for (size_t i = 0; i < rec.size();) {
    size_t j = i + 1;
    while (j < rec.size() && rec[j][0] == rec[i][0] && rec[j][1] == rec[i][1]) j++;
    for (size_t a = i; a < j; a++)
      for (size_t b = a + 1; b < j; b++) {
        int32_t t1 = rec[a][2], t2 = rec[b][2];
        if (t1 == t2) continue;
        pairs.push_back({std::min(t1, t2), std::max(t1, t2)});
      }
    i = j;
  }
  std::sort(pairs.begin(), pairs.end());
  pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
  c->adj_off.assign(nt + 1, 0);
  for (auto &p : pairs) {
    c->adj_off[p.first + 1]++;
    c->adj_off[p.second + 1]++;
  }
  for (int64_t t = 0; t < nt; t++) c->adj_off[t + 1] += c->adj_off[t];
  c->adj_nb.assign(c->adj_off[nt], 0);
  {
    std::vector<int32_t> cur(c->adj_off.begin(), c->adj_off.end() - 1);
    for (auto &p : pairs) {
      c->adj_nb[cur[p.first]++] = p.second;
      c->adj_nb[cur[p.second]++] = p.first;
    }
  }
  // basis slots
  std::vector<int32_t> slot_rwg(3 * nt, -1), slot_side(3 * nt, 0), rslot(2 * N);
  std::vector<int> cnt(nt, 0);
  for (int64_t m = 0; m < N; m++) {
    int32_t ts[2] = {c->h_tplus[m], c->h_tminus[m]};
    for (int s = 0; s < 2; s++) {
      int32_t t = ts[s];
      DMB_REQUIRE(cnt[t] < 3, DMB_ERR_ARGUMENT,
                  "RWG data assigns more than three basis functions to triangle " +
                      std::to_string(t + 1));
      slot_rwg[3 * t + cnt[t]] = (int32_t)m;
      slot_side[3 * t + cnt[t]] = s;
      rslot[2 * m + s] = 3 * t + cnt[t];
      cnt[t]++;
    }
  }
  // near records: self pairs and ordered adjacent pairs, canonical m <= n
  struct Key {
    int32_t m, n, ta, tb, ia, ib;
  };
  std::vector<Key> keys;
  keys.reserve(12 * nt);
  for (int64_t t = 0; t < nt; t++)
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        int32_t m = slot_rwg[3 * t + i], n = slot_rwg[3 * t + j];
        if (m < 0 || n < 0 || m > n) continue;
        keys.push_back({m, n, (int32_t)t, (int32_t)t, i, j});
      }
  for (int64_t ta = 0; ta < nt; ta++)
    for (int32_t q = c->adj_off[ta]; q < c->adj_off[ta + 1]; q++) {
      int32_t tb = c->adj_nb[q];
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
          int32_t m = slot_rwg[3 * ta + i], n = slot_rwg[3 * tb + j];
          if (m < 0 || n < 0 || m > n) continue;
          keys.push_back({m, n, (int32_t)ta, tb, i, j});
        }
    }
  std::sort(keys.begin(), keys.end(), [](const Key &a, const Key &b) {
    if (a.m != b.m) return a.m < b.m;
    if (a.n != b.n) return a.n < b.n;
    if (a.ta != b.ta) return a.ta < b.ta;
    if (a.tb != b.tb) return a.tb < b.tb;
    if (a.ia != b.ia) return a.ia < b.ia;
    return a.ib < b.ib;
  });
  std::vector<NearRec> recs(keys.size());
  std::vector<int2> ent;
  std::vector<int64_t> eoff;
  for (size_t i = 0; i < keys.size(); i++) {
    recs[i] = {keys[i].ta, keys[i].tb, keys[i].ia, keys[i].ib};
    if (i == 0 || keys[i].m != keys[i - 1].m || keys[i].n != keys[i - 1].n) {
      ent.push_back(make_int2(keys[i].m, keys[i].n));
      eoff.push_back((int64_t)i);
    }
  }
  eoff.push_back((int64_t)keys.size());
  c->n_near_rec = (int64_t)recs.size();
  c->n_near_entry = (int64_t)ent.size();

  auto up = [&](DevBuf &b, const void *src, size_t bytes) {
    b.ensure(bytes ? bytes : 16);
    if (bytes) DMB_CUDA(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, c->stream));
  };
  up(c->d_adj_off, c->adj_off.data(), c->adj_off.size() * 4);
  up(c->d_adj_nb, c->adj_nb.data(), c->adj_nb.size() * 4);
  up(c->d_rwg_slot, rslot.data(), rslot.size() * 4);
  // per RWG row: the near entries that touch it (as m or as n), in entry
  // order, with the other index
  std::vector<int64_t> roff(N + 1, 0);
  for (auto &e : ent) {
    roff[e.x + 1]++;
    if (e.x != e.y) roff[e.y + 1]++;
  }
  for (int64_t m = 0; m < N; m++) roff[m + 1] += roff[m];
  std::vector<int32_t> rent(roff[N]), rcol(roff[N]);
  {
    std::vector<int64_t> cur(roff.begin(), roff.end() - 1);
    for (size_t e = 0; e < ent.size(); e++) {
      const int32_t m = ent[e].x, n = ent[e].y;
      rent[cur[m]] = (int32_t)e;
      rcol[cur[m]++] = n;
      if (m != n) {
        rent[cur[n]] = (int32_t)e;
        rcol[cur[n]++] = m;
      }
    }
  }
  up(c->d_near_rec, recs.data(), recs.size() * sizeof(NearRec));
  up(c->d_near_entry_mn, ent.data(), ent.size() * sizeof(int2));
  up(c->d_near_entry_off, eoff.data(), eoff.size() * sizeof(int64_t));
  up(c->d_near_row_off, roff.data(), roff.size() * sizeof(int64_t));
  up(c->d_near_row_ent, rent.data(), rent.size() * 4);
  up(c->d_near_row_col, rcol.data(), rcol.size() * 4);
  c->d_near_entry_sum.ensure(std::max<size_t>(16, ent.size() * sizeof(double2)));
  c->d_near_val.ensure(std::max<size_t>(16, recs.size() * sizeof(double2)));
  up(c->d_slot_rwg, slot_rwg.data(), slot_rwg.size() * 4);
  up(c->d_slot_side, slot_side.data(), slot_side.size() * 4);
  c->d_tcache.ensure(sizeof(TriCache) * std::max<int64_t>(nt, 1));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  c->cache_valid = false;
}

void ensure_cache(dmb_ctx *c, int quad_order) {
  DMB_REQUIRE(c->have_mesh && c->have_rwg, DMB_ERR_STATE, "mesh and RWG data must be uploaded first");
  if (c->cache_valid && c->cache_quad_order == quad_order) return;
  QuadConst qc{};
  int nq = quad_rule(quad_order, qc.x1, qc.x2, qc.w);
  DMB_REQUIRE(nq > 0, DMB_ERR_ARGUMENT,
              "Unsupported quadrature order " + std::to_string(quad_order) + ". Use 1, 3, 4, or 7.");
  quad_rule(7, qc.h1, qc.h2, qc.wh);
  qc.nq = nq;
  c->nq = nq;
  for (int i = 0; i < 7; i++) {
    c->wq[i] = qc.w[i];
    c->wqh[i] = qc.wh[i];
    c->xi1[i] = qc.x1[i];
    c->xi2[i] = qc.x2[i];
    c->xh1[i] = qc.h1[i];
    c->xh2[i] = qc.h2[i];
  }
  double t0 = now_ms();
  const int64_t nt = c->nt;
  const int *slot = c->d_slot_rwg.as<int>();
  const int *side = c->d_slot_side.as<int>();
  const double *len = c->d_len.as<double>();
  const double *ap = c->d_ap.as<double>();
  const double *am = c->d_am.as<double>();
  const int *vpo = c->d_vpo.as<int>();
  const int *vmo = c->d_vmo.as<int>();
  DMB_LAUNCH(c, k_tri_cache, (unsigned)((nt + 127) / 128), 128, 0, (int)nt, c->d_xyz.as<double>(),
             c->d_tri.as<int>(), slot, side, len, ap, am, vpo, vmo, qc, c->d_tcache.as<TriCache>());
  c->d_centers.ensure(sizeof(double) * 3 * std::max<int64_t>(c->n, 1));
  DMB_LAUNCH(c, k_rwg_centers, (unsigned)((c->n + 127) / 128), 128, 0, (int)c->n,
             c->d_tcache.as<TriCache>(), c->d_tplus.as<int>(), c->d_tminus.as<int>(),
             c->d_centers.as<double>());
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  c->tm.geometry_ms = now_ms() - t0;
  double hw[14];
  for (int i = 0; i < 7; i++) {
    hw[i] = c->wq[i];
    hw[7 + i] = c->wqh[i];
  }
  c->d_wq.ensure(sizeof(hw));
  DMB_CUDA(cudaMemcpyAsync(c->d_wq.p, hw, sizeof(hw), cudaMemcpyHostToDevice, c->stream));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  c->cache_valid = true;
  c->cache_quad_order = quad_order;
  c->cache_gen++;
}

// value of every near record (self / edge-adjacent term per slot pair)
void near_values(dmb_ctx *c, double k, double inv_k2) {
  if (c->n_near_rec == 0) return;
  const double *dwq = c->d_wq.as<double>();
  DMB_LAUNCH(c, k_near_values, (unsigned)((c->n_near_rec + 127) / 128), 128, 0, c->n_near_rec,
             c->d_near_rec.as<NearRec>(), c->d_tcache.as<TriCache>(), c->nq, dwq, dwq + 7, k, inv_k2,
             c->d_near_val.as<double2>());
}

// EFIE prefactors with the reference's argument checks (EFIE.jl:699-720)
static void prefactors(double k, double eta0, int precision, double &inv_k2, double &omega_mu0) {
  DMB_REQUIRE(std::isfinite(k) && k != 0.0, DMB_ERR_ARGUMENT,
              "EFIE wavenumber must be finite and nonzero, got " + std::to_string(k));
  DMB_REQUIRE(std::isfinite(eta0) && eta0 != 0.0, DMB_ERR_ARGUMENT,
              "EFIE eta0 must be numeric, finite, and nonzero");
  DMB_REQUIRE(precision == DMB_PREC_FP64 || precision == DMB_PREC_MIXED, DMB_ERR_ARGUMENT,
              "precision must be DMB_PREC_FP64 or DMB_PREC_MIXED");
  double k2 = k * k;
  DMB_REQUIRE(std::isfinite(k2) && k2 != 0.0, DMB_ERR_OVERFLOW,
              "EFIE wavenumber squared is not representable");
  inv_k2 = 1.0 / k2;
  omega_mu0 = k * eta0;
  DMB_REQUIRE(std::isfinite(omega_mu0) && omega_mu0 != 0.0, DMB_ERR_OVERFLOW,
              "EFIE k*eta0 prefactor is not representable");
}

static void mark_assembled(dmb_ctx *c, double k, double eta0, int precision) {
  c->z_prec = precision;
  c->z_valid = true;
  c->op_kind = 0;  // the dense Z is the operator again
  c->z_version++;
  c->k = k;
  c->eta0 = eta0;
  c->pc_valid = false;
}

void assemble(dmb_ctx *c, double k, double eta0, int quad_order, int precision) {
  double inv_k2, omega_mu0;
  prefactors(k, eta0, precision, inv_k2, omega_mu0);
  ensure_cache(c, quad_order);
  double t0 = now_ms();
  const int64_t N = c->n;
  const bool f64 = precision == DMB_PREC_FP64;
  size_t esz = f64 ? sizeof(double2) : sizeof(float2);
  c->d_Z.ensure((size_t)std::max<int64_t>(N, 1) * std::max<int64_t>(N, 1) * esz);
  DMB_REQUIRE(c->nq == 1 || c->nq == 3 || c->nq == 4 || c->nq == 7, DMB_ERR_ARGUMENT,
              "unsupported quadrature size");
  // far triangle pairs straight into Z by RWG tiles (dmb_fartile.cu)
  const int T = far_tile_width(c, f64, k, inv_k2, omega_mu0);
  far_tiles(c, T, f64, k, inv_k2, omega_mu0);
  // near-singular records (always FP64)
  if (c->n_near_rec > 0) {
    near_values(c, k, inv_k2);
    if (f64)
      DMB_LAUNCH(c, k_near_add<double2>, (unsigned)((c->n_near_entry + 255) / 256), 256, 0,
                 c->n_near_entry, c->d_near_entry_mn.as<int2>(), c->d_near_entry_off.as<int64_t>(),
                 c->d_near_val.as<double2>(), omega_mu0, N, c->d_Z.as<double2>());
    else
      DMB_LAUNCH(c, k_near_add<float2>, (unsigned)((c->n_near_entry + 255) / 256), 256, 0,
                 c->n_near_entry, c->d_near_entry_mn.as<int2>(), c->d_near_entry_off.as<int64_t>(),
                 c->d_near_val.as<double2>(), omega_mu0, N, c->d_Z.as<float2>());
  }
  DMB_REQUIRE(far_error_word(c, f64) == 0, DMB_ERR_TIMEOUT, "assembly: a far-pair panel copy wait expired");
  c->tm.assembly_ms = now_ms() - t0;
  mark_assembled(c, k, eta0, precision);
}

double assemble_batch(const std::vector<dmb_ctx *> &cs, double k, double eta0, int quad_order, int precision,
                      BatchAsmBufs &bufs) {
  if (cs.empty()) return 0.0;
  double inv_k2, omega_mu0;
  prefactors(k, eta0, precision, inv_k2, omega_mu0);
  const bool f64 = precision == DMB_PREC_FP64;
  const size_t esz = f64 ? sizeof(double2) : sizeof(float2);
  dmb_ctx *big = cs[0], *c0 = cs[0];
  for (dmb_ctx *c : cs) {
    ensure_cache(c, quad_order);
    c->d_Z.ensure((size_t)std::max<int64_t>(c->n, 1) * std::max<int64_t>(c->n, 1) * esz);
    if (c->n > big->n) big = c;
  }
  // tile width of the largest surface's size bucket (autotuned there)
  const int T = far_tile_width(big, f64, k, inv_k2, omega_mu0);
  for (dmb_ctx *c : cs) c->far_tile_used = T;
  cudaEvent_t e0, e1;
  DMB_CUDA(cudaEventCreate(&e0));
  DMB_CUDA(cudaEventCreate(&e1));
  DMB_CUDA(cudaEventRecord(e0, c0->stream));
  far_tiles_batched(cs, T, f64, k, inv_k2, omega_mu0, bufs.far_jobs, bufs.far_tasks, bufs.far_err);
  std::vector<NearJob> jobs;
  int64_t nrec = 0, nent = 0;
  for (dmb_ctx *c : cs) {
    if (c->n_near_rec == 0) continue;
    NearJob jb;
    jb.recs = c->d_near_rec.as<NearRec>();
    jb.tc = c->d_tcache.as<TriCache>();
    jb.wq = c->d_wq.as<double>();
    jb.vals = c->d_near_val.as<double2>();
    jb.mn = c->d_near_entry_mn.as<int2>();
    jb.eoff = c->d_near_entry_off.as<int64_t>();
    jb.Z = c->d_Z.p;
    jb.N = c->n;
    jb.rec0 = nrec;
    jb.ent0 = nent;
    jb.k = k;
    jb.inv_k2 = inv_k2;
    jb.omega_mu0 = omega_mu0;
    jb.nq = c->nq;
    jobs.push_back(jb);
    nrec += c->n_near_rec;
    nent += c->n_near_entry;
  }
  if (!jobs.empty()) {
    bufs.near_jobs.ensure(jobs.size() * sizeof(NearJob));
    DMB_CUDA(cudaMemcpyAsync(bufs.near_jobs.p, jobs.data(), jobs.size() * sizeof(NearJob), cudaMemcpyHostToDevice,
                             c0->stream));
    const int nj = (int)jobs.size();
    DMB_LAUNCH(c0, k_near_values_batched, (unsigned)((nrec + 127) / 128), 128, 0, bufs.near_jobs.as<NearJob>(), nj,
               nrec);
    if (f64)
      DMB_LAUNCH(c0, k_near_add_batched<double2>, (unsigned)((nent + 255) / 256), 256, 0,
                 bufs.near_jobs.as<NearJob>(), nj, nent);
    else
      DMB_LAUNCH(c0, k_near_add_batched<float2>, (unsigned)((nent + 255) / 256), 256, 0,
                 bufs.near_jobs.as<NearJob>(), nj, nent);
  }
  DMB_CUDA(cudaEventRecord(e1, c0->stream));
  DMB_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  DMB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  unsigned err = 0;
  DMB_CUDA(cudaMemcpy(&err, bufs.far_err.p, 4, cudaMemcpyDeviceToHost));
  DMB_REQUIRE(err == 0, DMB_ERR_TIMEOUT, "batched assembly: a far-pair panel copy wait expired");
  for (dmb_ctx *c : cs) {
    c->tm.assembly_ms = ms;
    mark_assembled(c, k, eta0, precision);
  }
  return ms;
}

}  // namespace dmb
