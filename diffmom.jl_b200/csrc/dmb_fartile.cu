// dmb_fartile.cu -- the far triangle-pair part of the impedance matrix,
// written straight into Z by tiles of RWG functions.
//
// Reference: assemble_Z_efie (src/assembly/EFIE.jl:699-753) sums, for every
// RWG pair (m, n), the four triangle pairs of their supports (_efie_entry,
// EFIE.jl:439-512) with the product quadrature rule; a pair that is one
// triangle or shares an edge takes the singular path instead (here added
// afterwards from the near records, k_near_add in dmb_assemble.cu).
//
// Work unit: one CTA per (row tile I, column tile J), I <= J, of T x T RWG
// functions.  The triangles that carry a tile's functions (at most 2T) are
// packed once per mesh into a panel -- structure of arrays, 16-byte aligned,
// one per tile -- and each CTA stages its two panels into shared memory with
// the bulk-copy engine (cp.async.bulk completing on an mbarrier, bounded
// wait).
//   phase 1  the CTA's threads stride over the triangle pairs (a, b) of the two panels: the
//            quadrature points come from shared memory into registers, the
//            Nq x Nq moments of the Green function are formed and contracted
//            into the 3 x 3 block of the two triangles' basis slots; a slot
//            whose function lies in the tile lands in the tile's slot matrix
//            S[2 m' + side(m)][2 n' + side(n)] (shared memory).
//   phase 2  Z[m][n] = -i omega mu0 ((S++ + S--) + (S+- + S-+)), the four
//            triangle pairs of (m, n) summed in this fixed order, stored row by
//            row into the Z[I][J] block and, for I < J, column by column into
//            Z[J][I] (both coalesced).  The order is symmetric in (m, n), so Z
//            is bitwise symmetric; no slot matrix in HBM, no atomics.
// Triangles shared by neighbouring tiles are evaluated once per tile that
// holds them (about 2.3x the minimal pair count on sorted-edge RWG orders);
// in exchange the kernel writes Z once and reads nothing else from HBM.
//
// The FP64 flavour follows the reference's arithmetic (R from the global
// quadrature points); the FP32 flavour (mixed precision) takes R from the
// centroid difference rounded from FP64 plus FP32 local offsets.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <type_traits>

#include "dmb_device.cuh"
#include "dmb_internal.h"
#include "dmb_tcgen05.cuh"

namespace {

using dmb_tc::smem_u32;

// Panel of one RWG tile: P = 2T triangle entries, fields as arrays over the
// entries.  R is the arithmetic type of the flavour.
template <int NQ, int P, bool F64>
struct Panel {
  typedef typename std::conditional<F64, double, float>::type R;
  static constexpr int RS = (int)sizeof(R);
  static constexpr int OFF_CEN = 0;                        // double [3][P] centroid
  static constexpr int OFF_Q = OFF_CEN + 3 * P * 8;        // R [NQ][3][P] points (FP64 global, FP32 local)
  static constexpr int OFF_W = OFF_Q + 3 * NQ * P * RS;    // R [NQ][P] weight x 2A
  static constexpr int OFF_S = OFF_W + NQ * P * RS;        // R [3][P] signed basis scale
  static constexpr int OFF_DV = OFF_S + 3 * P * RS;        // R [3][P] surface divergence
  static constexpr int OFF_PL = OFF_DV + 3 * P * RS;       // R [3][3][P] opposite vertex - centroid
  static constexpr int OFF_TRI = OFF_PL + 9 * P * RS;      // int [P] triangle (-1: empty entry)
  static constexpr int OFF_NB = OFF_TRI + P * 4;           // int [3][P] edge neighbours (-1: none)
  static constexpr int OFF_SLOT = OFF_NB + 3 * P * 4;      // int [3][P] tile slot of each basis slot (-1: outside)
  static constexpr int OFF_MORE = OFF_SLOT + 3 * P * 4;    // int [P] 1: more than 3 neighbours (check the CSR)
  static constexpr int BYTES = (OFF_MORE + P * 4 + 15) / 16 * 16;
  static_assert(P % 4 == 0, "panel entries must keep 16-byte field alignment");
};

struct FarJob {
  const unsigned char *panels;  // ntiles panels
  const int *cnt;               // triangles per tile
  const int *aoff, *anb;        // edge adjacency of the surface's triangles (CSR)
  void *Z;                      // N x N row-major (complex128 or complex64)
  int64_t N;
  double k, inv_k2, omega_mu0;
};

constexpr long long FAR_WAIT_LIMIT = 1LL << 22;

__device__ __forceinline__ bool bar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool bar_wait_bounded(uint32_t bar) {
  for (long long it = 0; it < FAR_WAIT_LIMIT; it++)
    if (bar_try(bar, 0)) return true;
  return false;
}
// global -> shared bulk copy (16-byte aligned addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(bar)
               : "memory");
}

__device__ __forceinline__ bool csr_adjacent(const int *__restrict__ off, const int *__restrict__ nb, int ta, int tb) {
  for (int i = off[ta]; i < off[ta + 1]; i++)
    if (nb[i] == tb) return true;
  return false;
}

// sin(kR), cos(kR) from those of k Rc and the Taylor series of the short
// remainder d = k (R - Rc); a remainder above 0.75 (coarse meshes) takes the
// direct evaluation.  Series terms through d^16 / d^17: the first omitted
// term is below 1e-18 at |d| = 0.75.
__device__ __forceinline__ void phase_exp(double k, double R, double Rc, double s0, double c0, double &sn,
                                          double &cs) {
  const double d = k * (R - Rc);
  if (fabs(d) > 0.75) {
    sincos(k * R, &sn, &cs);
    return;
  }
  const double u = d * d;
  double cd = 1.0 / 20922789888000.0;  // 1/16!
  cd = fma(cd, u, -1.0 / 87178291200.0);
  cd = fma(cd, u, 1.0 / 479001600.0);
  cd = fma(cd, u, -1.0 / 3628800.0);
  cd = fma(cd, u, 1.0 / 40320.0);
  cd = fma(cd, u, -1.0 / 720.0);
  cd = fma(cd, u, 1.0 / 24.0);
  cd = fma(cd, u, -0.5);
  cd = fma(cd, u, 1.0);
  double sd = 1.0 / 355687428096000.0;  // 1/17!
  sd = fma(sd, u, -1.0 / 1307674368000.0);
  sd = fma(sd, u, 1.0 / 6227020800.0);
  sd = fma(sd, u, -1.0 / 39916800.0);
  sd = fma(sd, u, 1.0 / 362880.0);
  sd = fma(sd, u, -1.0 / 5040.0);
  sd = fma(sd, u, 1.0 / 120.0);
  sd = fma(sd, u, -1.0 / 6.0);
  sd = fma(sd, u, 1.0);
  sd *= d;
  // angle sum: (c0 + i s0)(cd + i sd)
  cs = fma(c0, cd, -s0 * sd);
  sn = fma(s0, cd, c0 * sd);
}

template <class SC>
__device__ __forceinline__ double2 tile_entry(const SC *S, int lds, int a, int b) {
  const SC *r0 = S + (2 * a) * lds + 2 * b;
  const SC *r1 = r0 + lds;
  double2 pp = to_d2(r0[0]), pm = to_d2(r0[1]), mp = to_d2(r1[0]), mm = to_d2(r1[1]);
  return make_double2((pp.x + mm.x) + (pm.x + mp.x), (pp.y + mm.y) + (pm.y + mp.y));
}

// CTA size: 256 threads for the FP32 flavour (80 registers, several CTAs per
// SM); 192 for the FP64 flavour, whose ~160 registers per thread would allow
// only one 256-thread CTA per SM -- two 192-thread CTAs keep 12 warps resident.
template <bool F64> struct FarThreads { static constexpr int value = F64 ? 192 : 256; };

template <int NQ, int T, bool F64>
__global__ void __launch_bounds__(FarThreads<F64>::value, F64 ? 2 : 3)
    k_far_tile(const FarJob *__restrict__ jobs, const int4 *__restrict__ tasks, unsigned *err) {
  constexpr int P = 2 * T, LDS = 2 * T;
  typedef Panel<NQ, P, F64> L;
  typedef typename L::R R;
  typedef typename std::conditional<F64, double2, float2>::type SC;
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ __align__(8) uint64_t bar;

  const int4 task = tasks[blockIdx.x];
  const FarJob jb = jobs[task.x];
  const int I = task.y, J = task.z;
  const bool diag = I == J;
  unsigned char *pa = sm;
  unsigned char *pb = diag ? sm : sm + L::BYTES;
  SC *S = reinterpret_cast<SC *>(sm + 2 * L::BYTES);
  const uint32_t b = smem_u32(&bar);
  if (threadIdx.x == 0) {
    dmb_tc::mbar_init(b, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    dmb_tc::mbar_expect_tx(b, diag ? L::BYTES : 2 * L::BYTES);
    bulk_g2s(smem_u32(pa), jb.panels + (size_t)I * L::BYTES, L::BYTES, b);
    if (!diag) bulk_g2s(smem_u32(pb), jb.panels + (size_t)J * L::BYTES, L::BYTES, b);
  }
  const int ua = jb.cnt[I], ub = jb.cnt[J];
  const bool ok = __syncthreads_and(bar_wait_bounded(b));
  if (!ok) {
    // the copies may still be in flight: wait for them (bounded) before the
    // CTA leaves, report, and write nothing
    if (threadIdx.x == 0) atomicOr(err, 1u);
    bar_wait_bounded(b);
    return;
  }

  const double *cenA = reinterpret_cast<const double *>(pa + L::OFF_CEN);
  const double *cenB = reinterpret_cast<const double *>(pb + L::OFF_CEN);
  const R *qA = reinterpret_cast<const R *>(pa + L::OFF_Q), *qB = reinterpret_cast<const R *>(pb + L::OFF_Q);
  const R *wA = reinterpret_cast<const R *>(pa + L::OFF_W), *wB = reinterpret_cast<const R *>(pb + L::OFF_W);
  const R *sA = reinterpret_cast<const R *>(pa + L::OFF_S), *sB = reinterpret_cast<const R *>(pb + L::OFF_S);
  const R *dA = reinterpret_cast<const R *>(pa + L::OFF_DV), *dB = reinterpret_cast<const R *>(pb + L::OFF_DV);
  const R *plA = reinterpret_cast<const R *>(pa + L::OFF_PL), *plB = reinterpret_cast<const R *>(pb + L::OFF_PL);
  const int *triA = reinterpret_cast<const int *>(pa + L::OFF_TRI);
  const int *triB = reinterpret_cast<const int *>(pb + L::OFF_TRI);
  const int *nbA = reinterpret_cast<const int *>(pa + L::OFF_NB);
  const int *slA = reinterpret_cast<const int *>(pa + L::OFF_SLOT);
  const int *slB = reinterpret_cast<const int *>(pb + L::OFF_SLOT);
  const int *moreA = reinterpret_cast<const int *>(pa + L::OFF_MORE);

  // ---- phase 1: triangle pairs -> tile slot matrix ----------------------
  // thread -> pairs p = tid, tid + blockDim, ... as (ia, ib) = (p / ub, p % ub),
  // stepped without a division per pair
  const int dq = blockDim.x / ub, dr = blockDim.x - dq * ub;
  int ia = threadIdx.x / ub, ib = threadIdx.x - (threadIdx.x / ub) * ub;
  for (; ia < ua; ia += dq, ib += dr, ia += (ib >= ub) ? 1 : 0, ib -= (ib >= ub) ? ub : 0) {
    const int ta = triA[ia], tb = triB[ib];
    const int rs[3] = {slA[ia], slA[P + ia], slA[2 * P + ia]};
    const int cs[3] = {slB[ib], slB[P + ib], slB[2 * P + ib]};
    bool near = ta == tb || nbA[ia] == tb || nbA[P + ia] == tb || nbA[2 * P + ia] == tb;
    if (!near && moreA[ia]) near = csr_adjacent(jb.aoff, jb.anb, ta, tb);
    if (near) {
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++)
          if (rs[i] >= 0 && cs[j] >= 0) S[rs[i] * LDS + cs[j]] = SC{};
      continue;
    }
    R m0r = 0, m0i = 0, mar[3] = {0, 0, 0}, mai[3] = {0, 0, 0}, mbr[3] = {0, 0, 0}, mbi[3] = {0, 0, 0}, mabr = 0,
      mabi = 0;
    if constexpr (F64) {
      const double k = jb.k;
      const double ca0 = cenA[ia], ca1 = cenA[P + ia], ca2 = cenA[2 * P + ia];
      const double cb0 = cenB[ib], cb1 = cenB[P + ib], cb2 = cenB[2 * P + ib];
      // phase of the centroid distance, once per pair: exp(-ik R) =
      // exp(-ik Rc) exp(-ik (R - Rc)) with the short second factor from
      // its Taylor series (|k (R - Rc)| <= 0.75: truncation below 1e-18)
      const double cdx = ca0 - cb0, cdy = ca1 - cb1, cdz = ca2 - cb2;
      const double Rc = sqrt(cdx * cdx + cdy * cdy + cdz * cdz);
      double s0, c0;
      sincos(k * Rc, &s0, &c0);
#pragma unroll
      for (int bq = 0; bq < NQ; bq++) {
        const double qb0 = qB[(3 * bq + 0) * P + ib], qb1 = qB[(3 * bq + 1) * P + ib],
                     qb2 = qB[(3 * bq + 2) * P + ib];
        const double lb0 = qb0 - cb0, lb1 = qb1 - cb1, lb2 = qb2 - cb2;
        const double wb = wB[bq * P + ib];
#pragma unroll
        for (int aq = 0; aq < NQ; aq++) {
          const double qa0 = qA[(3 * aq + 0) * P + ia], qa1 = qA[(3 * aq + 1) * P + ia],
                       qa2 = qA[(3 * aq + 2) * P + ia];
          const double la0 = qa0 - ca0, la1 = qa1 - ca1, la2 = qa2 - ca2;
          const double wa = wA[aq * P + ia];
          double dx = qa0 - qb0, dy = qa1 - qb1, dz = qa2 - qb2;
          const double R2 = dx * dx + dy * dy + dz * dz;
          const double rinv = rsqrt(R2);
          const double Rr = R2 * rinv;
          double sn, cs_;
          phase_exp(k, Rr, Rc, s0, c0, sn, cs_);
          double g = (DMB_INV_FOUR_PI * rinv) * (wa * wb);
          double gr = cs_ * g, gi = -sn * g;  // exp(-ikR)/(4 pi R) * W
          m0r += gr;
          m0i += gi;
          mar[0] = fma(gr, la0, mar[0]); mai[0] = fma(gi, la0, mai[0]);
          mar[1] = fma(gr, la1, mar[1]); mai[1] = fma(gi, la1, mai[1]);
          mar[2] = fma(gr, la2, mar[2]); mai[2] = fma(gi, la2, mai[2]);
          mbr[0] = fma(gr, lb0, mbr[0]); mbi[0] = fma(gi, lb0, mbi[0]);
          mbr[1] = fma(gr, lb1, mbr[1]); mbi[1] = fma(gi, lb1, mbi[1]);
          mbr[2] = fma(gr, lb2, mbr[2]); mbi[2] = fma(gi, lb2, mbi[2]);
          double dd = la0 * lb0 + la1 * lb1 + la2 * lb2;
          mabr = fma(gr, dd, mabr);
          mabi = fma(gi, dd, mabi);
        }
      }
    } else {
      const float k = (float)jb.k;
      const float dc0 = (float)(cenA[ia] - cenB[ib]), dc1 = (float)(cenA[P + ia] - cenB[P + ib]),
                  dc2 = (float)(cenA[2 * P + ia] - cenB[2 * P + ib]);
      const float c4pi = 0.0795774715f;
#pragma unroll
      for (int bq = 0; bq < NQ; bq++) {
        const float lb0 = qB[(3 * bq + 0) * P + ib], lb1 = qB[(3 * bq + 1) * P + ib],
                    lb2 = qB[(3 * bq + 2) * P + ib];
        const float wb = wB[bq * P + ib];
#pragma unroll
        for (int aq = 0; aq < NQ; aq++) {
          const float la0 = qA[(3 * aq + 0) * P + ia], la1 = qA[(3 * aq + 1) * P + ia],
                      la2 = qA[(3 * aq + 2) * P + ia];
          const float wa = wA[aq * P + ia];
          float dx = dc0 + (la0 - lb0), dy = dc1 + (la1 - lb1), dz = dc2 + (la2 - lb2);
          float R2 = dx * dx + dy * dy + dz * dz;
          float rinv = rsqrtf(R2);
          float Rr = R2 * rinv;
          float sn, cs_;
          sincosf(k * Rr, &sn, &cs_);
          float g = (c4pi * rinv) * (wa * wb);
          float gr = cs_ * g, gi = -sn * g;
          m0r += gr;
          m0i += gi;
          mar[0] = fmaf(gr, la0, mar[0]); mai[0] = fmaf(gi, la0, mai[0]);
          mar[1] = fmaf(gr, la1, mar[1]); mai[1] = fmaf(gi, la1, mai[1]);
          mar[2] = fmaf(gr, la2, mar[2]); mai[2] = fmaf(gi, la2, mai[2]);
          mbr[0] = fmaf(gr, lb0, mbr[0]); mbi[0] = fmaf(gi, lb0, mbi[0]);
          mbr[1] = fmaf(gr, lb1, mbr[1]); mbi[1] = fmaf(gi, lb1, mbi[1]);
          mbr[2] = fmaf(gr, lb2, mbr[2]); mbi[2] = fmaf(gi, lb2, mbi[2]);
          float dd = la0 * lb0 + la1 * lb1 + la2 * lb2;
          mabr = fmaf(gr, dd, mabr);
          mabi = fmaf(gi, dd, mabi);
        }
      }
    }
    const R inv_k2 = (R)jb.inv_k2;
    // block(i, j) = s_i s_j [Mab - Ma.pj' - Mb.pi' + (pi'.pj') M0] - dv_i dv_j M0 / k^2
#pragma unroll
    for (int i = 0; i < 3; i++) {
      if (rs[i] < 0) continue;
      const R si = sA[i * P + ia], dvi = dA[i * P + ia];
      const R pi0 = plA[(3 * i + 0) * P + ia], pi1 = plA[(3 * i + 1) * P + ia], pi2 = plA[(3 * i + 2) * P + ia];
      const R mbpr = mbr[0] * pi0 + mbr[1] * pi1 + mbr[2] * pi2;
      const R mbpi = mbi[0] * pi0 + mbi[1] * pi1 + mbi[2] * pi2;
#pragma unroll
      for (int j = 0; j < 3; j++) {
        if (cs[j] < 0) continue;
        const R sj = sB[j * P + ib], dvj = dB[j * P + ib];
        const R pj0 = plB[(3 * j + 0) * P + ib], pj1 = plB[(3 * j + 1) * P + ib], pj2 = plB[(3 * j + 2) * P + ib];
        const R mapr = mar[0] * pj0 + mar[1] * pj1 + mar[2] * pj2;
        const R mapi = mai[0] * pj0 + mai[1] * pj1 + mai[2] * pj2;
        const R pp = pi0 * pj0 + pi1 * pj1 + pi2 * pj2;
        const R ss = si * sj, sc = dvi * dvj * inv_k2;
        SC v;
        v.x = ss * (mabr - mapr - mbpr + pp * m0r) - sc * m0r;
        v.y = ss * (mabi - mapi - mbpi + pp * m0i) - sc * m0i;
        S[rs[i] * LDS + cs[j]] = v;
      }
    }
  }
  __syncthreads();

  // ---- phase 2: Z entries of the tile (and its transpose) ---------------
  typedef SC ZC;
  ZC *Z = reinterpret_cast<ZC *>(jb.Z);
  const int64_t N = jb.N;
  const int mrows = (int)min((int64_t)T, N - (int64_t)I * T);
  const int ncols = (int)min((int64_t)T, N - (int64_t)J * T);
  const double om = jb.omega_mu0;
  for (int e = threadIdx.x; e < T * T; e += blockDim.x) {
    const int mi = e / T, nj = e - mi * T;
    if (mi >= mrows || nj >= ncols) continue;
    // diagonal tiles: both (m, n) and (n, m) from the entry with m <= n
    const int a = (diag && mi > nj) ? nj : mi, c = (diag && mi > nj) ? mi : nj;
    const double2 v = tile_entry(S, LDS, a, c);
    // (-i w mu0) (re + i im) = (w mu0 im, -w mu0 re)
    store_c(Z + ((int64_t)I * T + mi) * N + (int64_t)J * T + nj, make_double2(om * v.y, -om * v.x));
  }
  if (!diag) {
    for (int e = threadIdx.x; e < T * T; e += blockDim.x) {
      const int nj = e / T, mi = e - nj * T;
      if (mi >= mrows || nj >= ncols) continue;
      const double2 v = tile_entry(S, LDS, mi, nj);
      store_c(Z + ((int64_t)J * T + nj) * N + (int64_t)I * T + mi, make_double2(om * v.y, -om * v.x));
    }
  }
}

// One thread per (tile, panel entry): copy the entry's triangle from the
// per-triangle cache into the panel layout and resolve its slot targets.
template <int NQ, int P, bool F64>
__global__ void k_far_pack(int ntiles, int T, int64_t N, const int *__restrict__ tile_tri,
                           const TriCache *__restrict__ tc, const int *__restrict__ aoff, const int *__restrict__ anb,
                           unsigned char *__restrict__ panels) {
  typedef Panel<NQ, P, F64> L;
  typedef typename L::R R;
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (int64_t)ntiles * P) return;
  const int k = (int)(gid / P), t = (int)(gid % P);
  unsigned char *base = panels + (size_t)k * L::BYTES;
  double *cen = reinterpret_cast<double *>(base + L::OFF_CEN);
  R *q = reinterpret_cast<R *>(base + L::OFF_Q);
  R *w = reinterpret_cast<R *>(base + L::OFF_W);
  R *s = reinterpret_cast<R *>(base + L::OFF_S);
  R *dv = reinterpret_cast<R *>(base + L::OFF_DV);
  R *pl = reinterpret_cast<R *>(base + L::OFF_PL);
  int *tri = reinterpret_cast<int *>(base + L::OFF_TRI);
  int *nb = reinterpret_cast<int *>(base + L::OFF_NB);
  int *slot = reinterpret_cast<int *>(base + L::OFF_SLOT);
  int *more = reinterpret_cast<int *>(base + L::OFF_MORE);
  const int tr = tile_tri[gid];
  if (tr < 0) {
    for (int d = 0; d < 3; d++) cen[d * P + t] = 0.0;
    for (int i = 0; i < 3 * NQ; i++) q[i * P + t] = 0;
    for (int i = 0; i < NQ; i++) w[i * P + t] = 0;
    for (int i = 0; i < 3; i++) s[i * P + t] = dv[i * P + t] = 0;
    for (int i = 0; i < 9; i++) pl[i * P + t] = 0;
    tri[t] = -1;
    for (int i = 0; i < 3; i++) nb[i * P + t] = slot[i * P + t] = -1;
    more[t] = 0;
    return;
  }
  const TriCache &c = tc[tr];
  for (int d = 0; d < 3; d++) cen[d * P + t] = c.cen[d];
  for (int a = 0; a < NQ; a++) {
    for (int d = 0; d < 3; d++) q[(3 * a + d) * P + t] = F64 ? (R)c.qp[a][d] : (R)c.ql[a][d];
    w[a * P + t] = (R)c.w2a[a];
  }
  const int64_t lo = (int64_t)k * T, hi = std::min<int64_t>(N, lo + T);
  for (int i = 0; i < 3; i++) {
    s[i * P + t] = (R)c.s[i];
    dv[i * P + t] = (R)c.dv[i];
    for (int d = 0; d < 3; d++) pl[(3 * i + d) * P + t] = (R)c.pl[i][d];
    const int n = c.rwg[i];
    slot[i * P + t] = (n >= 0 && n >= lo && n < hi) ? (int)(2 * (n - lo) + c.side[i]) : -1;
  }
  tri[t] = tr;
  const int o0 = aoff[tr], o1 = aoff[tr + 1];
  const bool many = o1 - o0 > 3;
  for (int i = 0; i < 3; i++) nb[i * P + t] = (!many && o0 + i < o1) ? anb[o0 + i] : -1;
  more[t] = many ? 1 : 0;
}

template <int NQ, int T, bool F64>
size_t far_smem_bytes() {
  typedef Panel<NQ, 2 * T, F64> L;
  return 2 * (size_t)L::BYTES + (size_t)(2 * T) * (2 * T) * (F64 ? sizeof(double2) : sizeof(float2));
}

template <int NQ, int T, bool F64>
void far_launch_t(dmb_ctx *c, const FarJob *d_jobs, const int4 *d_tasks, int64_t ntasks, unsigned *err) {
  const size_t smem = far_smem_bytes<NQ, T, F64>();
  static std::once_flag once;
  std::call_once(once, [&] {
    cudaFuncSetAttribute(k_far_tile<NQ, T, F64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  });
  DMB_LAUNCH(c, (k_far_tile<NQ, T, F64>), (unsigned)ntasks, FarThreads<F64>::value, smem, d_jobs, d_tasks, err);
}

template <int NQ, int T, bool F64>
void far_pack_t(dmb_ctx *c, int ntiles, const int *tile_tri, unsigned char *panels) {
  constexpr int P = 2 * T;
  const int64_t n = (int64_t)ntiles * P;
  DMB_LAUNCH(c, (k_far_pack<NQ, P, F64>), (unsigned)((n + 127) / 128), 128, 0, ntiles, T, c->n, tile_tri,
             c->d_tcache.as<TriCache>(), c->d_adj_off.as<int>(), c->d_adj_nb.as<int>(), panels);
}

template <int NQ, int T, bool F64>
int panel_bytes_t() {
  return Panel<NQ, 2 * T, F64>::BYTES;
}

// dispatch over the runtime (nq, T, precision) to the instantiated shapes:
// FP64 T in {16, 32}, FP32 T in {32, 64}
template <class Fn>
void far_dispatch(int nq, int T, bool f64, Fn &&fn) {
#define FT_CASE(NQV, TV, FV)                                  \
  if (nq == NQV && T == TV && f64 == FV) {                    \
    fn(std::integral_constant<int, NQV>{}, std::integral_constant<int, TV>{}, std::integral_constant<bool, FV>{}); \
    return;                                                   \
  }
#define FT_NQ(NQV) FT_CASE(NQV, 16, true) FT_CASE(NQV, 32, true) FT_CASE(NQV, 32, false) FT_CASE(NQV, 64, false)
  FT_NQ(1)
  FT_NQ(3)
  FT_NQ(4)
  FT_NQ(7)
#undef FT_NQ
#undef FT_CASE
  throw DmbError{DMB_ERR_ARGUMENT, "far-pair tile: no kernel for quadrature size " + std::to_string(nq) +
                                       ", tile width " + std::to_string(T) + (f64 ? " (FP64)" : " (FP32)")};
}

}  // namespace

namespace dmb {

bool far_tile_width_valid(int T, bool f64) { return f64 ? (T == 16 || T == 32) : (T == 32 || T == 64); }

// Per-tile triangle lists (host, O(N log T)), then the panels on the device.
void far_panels(dmb_ctx *c, int T, bool f64) {
  FarTileState &st = c->ft[f64 ? 1 : 0];
  if (st.valid && st.T == T && st.nq == c->nq && st.cache_gen == c->cache_gen) return;
  DMB_REQUIRE(far_tile_width_valid(T, f64), DMB_ERR_ARGUMENT,
              "far-pair tile width must be " + std::string(f64 ? "16 or 32" : "32 or 64") + " for this precision");
  const int64_t N = c->n;
  const int P = 2 * T;
  const int ntiles = (int)((N + T - 1) / T);
  std::vector<int32_t> tile_tri((size_t)ntiles * P, -1), cnt(ntiles, 0);
  std::vector<int32_t> buf;
  buf.reserve(P);
  for (int k = 0; k < ntiles; k++) {
    buf.clear();
    const int64_t lo = (int64_t)k * T, hi = std::min<int64_t>(N, lo + T);
    for (int64_t m = lo; m < hi; m++) {
      buf.push_back(c->h_tplus[m]);
      buf.push_back(c->h_tminus[m]);
    }
    std::sort(buf.begin(), buf.end());
    buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
    cnt[k] = (int32_t)buf.size();
    std::copy(buf.begin(), buf.end(), tile_tri.begin() + (size_t)k * P);
  }
  int pbytes = 0;
  far_dispatch(c->nq, T, f64, [&](auto NQ, auto TT, auto FV) { pbytes = panel_bytes_t<decltype(NQ)::value, decltype(TT)::value, decltype(FV)::value>(); });
  DevBuf lists;
  lists.ensure(tile_tri.size() * 4);
  DMB_CUDA(cudaMemcpyAsync(lists.p, tile_tri.data(), tile_tri.size() * 4, cudaMemcpyHostToDevice, c->stream));
  st.d_cnt.ensure(cnt.size() * 4);
  DMB_CUDA(cudaMemcpyAsync(st.d_cnt.p, cnt.data(), cnt.size() * 4, cudaMemcpyHostToDevice, c->stream));
  st.d_panels.ensure((size_t)ntiles * pbytes);
  if (ntiles > 0)
    far_dispatch(c->nq, T, f64, [&](auto NQ, auto TT, auto FV) {
    far_pack_t<decltype(NQ)::value, decltype(TT)::value, decltype(FV)::value>(c, ntiles, lists.as<int>(), st.d_panels.as<unsigned char>());
  });
  // tasks: every tile pair I <= J, row by row
  std::vector<int4> tasks;
  tasks.reserve((size_t)ntiles * (ntiles + 1) / 2);
  for (int i = 0; i < ntiles; i++)
    for (int j = i; j < ntiles; j++) tasks.push_back(make_int4(0, i, j, 0));
  st.d_tasks.ensure(tasks.size() * sizeof(int4));
  DMB_CUDA(cudaMemcpyAsync(st.d_tasks.p, tasks.data(), tasks.size() * sizeof(int4), cudaMemcpyHostToDevice,
                           c->stream));
  st.d_job.ensure(sizeof(FarJob));
  st.d_err.ensure(16);
  DMB_CUDA(cudaStreamSynchronize(c->stream));  // `lists` is released on return
  st.ntasks = (int64_t)tasks.size();
  st.ntiles = ntiles;
  st.T = T;
  st.nq = c->nq;
  st.cache_gen = c->cache_gen;
  st.valid = true;
}

// Far part of Z (every entry; near triangle pairs contribute zero) on the
// context stream, for the tile width T.
void far_tiles(dmb_ctx *c, int T, bool f64, double k, double inv_k2, double omega_mu0) {
  far_panels(c, T, f64);
  FarTileState &st = c->ft[f64 ? 1 : 0];
  FarJob jb;
  jb.panels = st.d_panels.as<unsigned char>();
  jb.cnt = st.d_cnt.as<int>();
  jb.aoff = c->d_adj_off.as<int>();
  jb.anb = c->d_adj_nb.as<int>();
  jb.Z = c->d_Z.p;
  jb.N = c->n;
  jb.k = k;
  jb.inv_k2 = inv_k2;
  jb.omega_mu0 = omega_mu0;
  DMB_CUDA(cudaMemcpyAsync(st.d_job.p, &jb, sizeof(jb), cudaMemcpyHostToDevice, c->stream));
  DMB_CUDA(cudaMemsetAsync(st.d_err.p, 0, 4, c->stream));
  if (st.ntasks == 0) return;
  kt_begin(c);
  far_dispatch(c->nq, T, f64, [&](auto NQ, auto TT, auto FV) {
    far_launch_t<decltype(NQ)::value, decltype(TT)::value, decltype(FV)::value>(
        c, st.d_job.as<FarJob>(), st.d_tasks.as<int4>(), st.ntasks, st.d_err.as<unsigned>());
  });
  kt_end(c, (double)c->n * (double)c->n * (f64 ? 16.0 : 8.0), 5);
}

unsigned far_error_word(dmb_ctx *c, bool f64) {
  FarTileState &st = c->ft[f64 ? 1 : 0];
  if (!st.d_err.p) return 0;
  unsigned e = 0;
  DMB_CUDA(cudaMemcpyAsync(&e, st.d_err.p, 4, cudaMemcpyDeviceToHost, c->stream));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  return e;
}

// Tile-width autotuner: per (device, mesh-size bucket, precision, quadrature
// size) each candidate width is timed once with CUDA events on the context
// stream (after one untimed launch that builds its panels and loads the
// kernel) and the fastest is kept for the process.  DMB_OPT_FAR_TILE pins a
// width instead.  Every width writes the same Z bit for bit (the per-entry
// arithmetic does not depend on the tiling).
static std::mutex g_far_tune_mu;
static std::vector<std::pair<int64_t, int>> g_far_tune;  // (device, size bucket, precision, nq) -> width

static int64_t far_tune_key(int device, int64_t n, bool f64, int nq) {
  int bucket = 0;
  while ((int64_t)1 << (bucket + 1) <= n) bucket++;
  return ((int64_t)device << 24) | ((int64_t)bucket << 8) | ((f64 ? 1 : 0) << 4) | nq;
}

// The width the tuner already chose for a mesh of n RWG functions (or the
// context's pin), 0 if that bucket has not been timed yet.
int far_tile_width_known(dmb_ctx *c, int64_t n, bool f64) {
  if (c->far_tile > 0) return far_tile_width_valid(c->far_tile, f64) ? c->far_tile : 0;
  const int64_t key = far_tune_key(c->device, n, f64, c->nq);
  std::lock_guard<std::mutex> lk(g_far_tune_mu);
  for (auto &e : g_far_tune)
    if (e.first == key) return e.second;
  return 0;
}

int far_tile_width(dmb_ctx *c, bool f64, double k, double inv_k2, double omega_mu0) {
  if (c->far_tile > 0) {
    DMB_REQUIRE(far_tile_width_valid(c->far_tile, f64), DMB_ERR_ARGUMENT,
                "DMB_OPT_FAR_TILE must be " + std::string(f64 ? "16 or 32" : "32 or 64") + " for this precision");
    return c->far_tile_used = c->far_tile;
  }
  const int64_t key = far_tune_key(c->device, c->n, f64, c->nq);
  auto &mu = g_far_tune_mu;
  auto &table = g_far_tune;
  {
    std::lock_guard<std::mutex> lk(mu);
    for (auto &e : table)
      if (e.first == key) return c->far_tile_used = e.second;
  }
  const int cand[2] = {f64 ? 16 : 32, f64 ? 32 : 64};
  cudaEvent_t e0, e1;
  DMB_CUDA(cudaEventCreate(&e0));
  DMB_CUDA(cudaEventCreate(&e1));
  int best = cand[1];
  float best_ms = 0;
  for (int T : cand) {
    far_tiles(c, T, f64, k, inv_k2, omega_mu0);
    DMB_CUDA(cudaEventRecord(e0, c->stream));
    far_tiles(c, T, f64, k, inv_k2, omega_mu0);
    DMB_CUDA(cudaEventRecord(e1, c->stream));
    DMB_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    DMB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (best_ms == 0 || ms < best_ms) {
      best_ms = ms;
      best = T;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::lock_guard<std::mutex> lk(mu);
  table.push_back({key, best});
  return c->far_tile_used = best;
}

// Far part of Z for many surfaces in ONE launch (uneven surface batches):
// every surface's tile pairs in one task list, largest surface first, on the
// stream of cs[0] (the caller's batch stream).  The surfaces share the tile
// width T, the quadrature size and the precision; each has its own panels,
// adjacency, Z and wavenumber.  jobs / tasks / err: device buffers the caller
// keeps between calls.
void far_tiles_batched(const std::vector<dmb_ctx *> &cs, int T, bool f64, double k, double inv_k2,
                       double omega_mu0, DevBuf &d_jobs, DevBuf &d_tasks, DevBuf &d_err) {
  if (cs.empty()) return;
  dmb_ctx *c0 = cs[0];
  const int nq = cs[0]->nq;
  for (dmb_ctx *c : cs) {
    DMB_REQUIRE(c->nq == nq, DMB_ERR_ARGUMENT, "batched assembly needs one quadrature rule");
    far_panels(c, T, f64);
  }
  std::vector<FarJob> jobs(cs.size());
  std::vector<int> order(cs.size());
  for (size_t i = 0; i < cs.size(); i++) {
    FarTileState &st = cs[i]->ft[f64 ? 1 : 0];
    FarJob &jb = jobs[i];
    jb.panels = st.d_panels.as<unsigned char>();
    jb.cnt = st.d_cnt.as<int>();
    jb.aoff = cs[i]->d_adj_off.as<int>();
    jb.anb = cs[i]->d_adj_nb.as<int>();
    jb.Z = cs[i]->d_Z.p;
    jb.N = cs[i]->n;
    jb.k = k;
    jb.inv_k2 = inv_k2;
    jb.omega_mu0 = omega_mu0;
    order[i] = (int)i;
  }
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cs[a]->n > cs[b]->n; });
  std::vector<int4> tasks;
  for (int s : order) {
    const int nt = cs[s]->ft[f64 ? 1 : 0].ntiles;
    for (int i = 0; i < nt; i++)
      for (int j = i; j < nt; j++) tasks.push_back(make_int4(s, i, j, 0));
  }
  d_jobs.ensure(jobs.size() * sizeof(FarJob));
  d_tasks.ensure(std::max<size_t>(1, tasks.size()) * sizeof(int4));
  d_err.ensure(16);
  DMB_CUDA(cudaMemcpyAsync(d_jobs.p, jobs.data(), jobs.size() * sizeof(FarJob), cudaMemcpyHostToDevice, c0->stream));
  DMB_CUDA(cudaMemcpyAsync(d_tasks.p, tasks.data(), tasks.size() * sizeof(int4), cudaMemcpyHostToDevice,
                           c0->stream));
  DMB_CUDA(cudaMemsetAsync(d_err.p, 0, 4, c0->stream));
  if (tasks.empty()) return;
  far_dispatch(nq, T, f64, [&](auto NQ, auto TT, auto FV) {
    far_launch_t<decltype(NQ)::value, decltype(TT)::value, decltype(FV)::value>(
        c0, d_jobs.as<FarJob>(), d_tasks.as<int4>(), (int64_t)tasks.size(), d_err.as<unsigned>());
  });
  // the host vectors must outlive the asynchronous copies
  DMB_CUDA(cudaStreamSynchronize(c0->stream));
}

void far_release(dmb_ctx *c) {
  for (auto &st : c->ft) {
    DevBuf *b[] = {&st.d_panels, &st.d_cnt, &st.d_tasks, &st.d_job, &st.d_err};
    for (DevBuf *x : b) x->release();
    st.valid = false;
  }
}

}  // namespace dmb
