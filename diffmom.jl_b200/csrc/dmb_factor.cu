// dmb_factor.cu -- near-field preconditioner: extraction, factorisation, apply.
//
//   * extraction (NearFieldPreconditioner.jl:247-369, 429-464, 670-716):
//     Z_nf[m][n] = Z[m][n] when the RWG centres are within `cutoff`
//     (inclusive, exact tie-break), else 0; nnz counted for nnz_ratio.
//   * Jacobi (:623-668): 1 / z_ii with the 1e-10 * max|z_ii| floor.
//   * factorisation: Z_nf is complex symmetric (Z is, and the distance test is
//     symmetric), so it is factored as L D L^T -- unit lower L, diagonal D, no
//     pivoting -- which has the same inverse as the reference's UMFPACK LU up to
//     rounding, at half the flops.  Right-looking, panel width NB = 64:
//       k_ldlt_diag    one CTA factors the 64x64 diagonal block and writes the
//                      inverse of its unit-lower factor (used twice: by the panel
//                      and by the triangular solves);
//       k_ldlt_panel   L21 D1 = A21 L11^-T as a small GEMM with that inverse,
//                      L21 = (L21 D1) D1^-1, rows in parallel;
//       k_ldlt_update  trailing update A22 -= (L21 D1) L21^T on lower tiles
//                      (FP64 SIMT for complex128 factors, FP32 SIMT or the
//                      tensor-core kernel for complex64 factors); inside a
//                      256-wide panel its first CTA then factors the next
//                      diagonal block, so that block needs no launch of its own.
//     A zero or non-finite pivot stops with DMB_ERR_BREAKDOWN.
//   * apply (NearFieldOperator, :1034-1054): L y = x, z = y / D, L^T x = z as
//     one kernel per sweep.  Each CTA draws a ticket (block row, launch order),
//     accumulates the contributions of already-solved block rows in registers as
//     their flags appear, then multiplies by the precomputed inverse of its
//     diagonal block.  Every wait is bounded: on expiry the kernel sets an error
//     bit and returns; the host raises DMB_ERR_TIMEOUT.
#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstring>

#include "dmb_device.cuh"
#include "dmb_internal.h"

namespace dmb {
void tc_ldlt_update_c64(dmb_ctx *c, int64_t N, int64_t r0, int64_t c_hi, int64_t jcol, int K, float2 *F,
                        const float2 *W, int wstride, int woff, int slot);
}  // namespace dmb

namespace {

constexpr int NB = 64;                      // panel width == triangular-solve block
constexpr long long SPIN_LIMIT = 20000000;  // ~2-4 s with nanosleep

unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// ---------------------------------------------------------------------------
// near-field extraction
// ---------------------------------------------------------------------------
__device__ bool within_cutoff_exact(const double *a, const double *b, double cutoff) {
  // compare the exact squared distance with cutoff^2 in double-double
  double s = 0, e = 0;
  double v[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
  for (int i = 0; i < 3; i++) {
    double p = v[i] * v[i], pe = fma(v[i], v[i], -p);
    double t = s + p, bb = t - s;
    e += (s - (t - bb)) + (p - bb) + pe;
    s = t;
  }
  double c2 = cutoff * cutoff, c2e = fma(cutoff, cutoff, -c2);
  return (s - c2) + (e - c2e) <= 0.0;
}

// 32 x 32 tiles; centres staged in shared memory; the squared distance is
// compared with a band around cutoff^2 and only the band goes to the exact test
template <class ZC, class FC>
__global__ void __launch_bounds__(256) k_nf_mask(int64_t N, const ZC *__restrict__ Z, const double *__restrict__ cen,
                                                 double cutoff, FC *__restrict__ F,
                                                 unsigned long long *__restrict__ nnz) {
  __shared__ double cm[32][3], cn[32][3];
  int64_t m0 = (int64_t)blockIdx.y * 32, n0 = (int64_t)blockIdx.x * 32;
  int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  if (threadIdx.x < 96) {
    int i = threadIdx.x / 3, d = threadIdx.x % 3;
    cm[i][d] = (m0 + i < N) ? cen[3 * (m0 + i) + d] : 0.0;
    cn[i][d] = (n0 + i < N) ? cen[3 * (n0 + i) + d] : 0.0;
  }
  __syncthreads();
  const bool all_in = !isfinite(cutoff);
  const double c2 = cutoff * cutoff;
  const double lo = c2 * (1 - 1e-12), hi = c2 * (1 + 1e-12);
  unsigned keep_cnt = 0;
  int64_t n = n0 + tx;
  for (int i = ty; i < 32; i += 8) {
    int64_t m = m0 + i;
    if (m >= N || n >= N) continue;
    bool keep;
    if (all_in) keep = true;
    else if (cutoff <= 0.0) keep = (m == n);
    else {
      double dx = cm[i][0] - cn[tx][0], dy = cm[i][1] - cn[tx][1], dz = cm[i][2] - cn[tx][2];
      double d2 = dx * dx + dy * dy + dz * dz;
      keep = (m == n) || d2 < lo || (d2 <= hi && within_cutoff_exact(cm[i], cn[tx], cutoff));
    }
    store_c(F + m * N + n, keep ? to_d2(Z[m * N + n]) : make_double2(0, 0));
    keep_cnt += keep;
  }
  unsigned cnt = __reduce_add_sync(0xffffffffu, keep_cnt);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(nnz, (unsigned long long)cnt);
}

template <class ZC>
__global__ void k_diag_max(int64_t N, const ZC *__restrict__ Z, double *__restrict__ out, unsigned *__restrict__ bad) {
  __shared__ double red[32];
  double mx = 0;
  for (int64_t i = threadIdx.x; i < N; i += blockDim.x) {
    double2 z = to_d2(Z[i * N + i]);
    double a = hypot(z.x, z.y);
    if (!isfinite(a)) atomicOr(bad, 1u);
    mx = fmax(mx, a);
  }
  mx = warp_max(mx);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32] = mx;
  __syncthreads();
  if (threadIdx.x < 32) {
    mx = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : 0;
    mx = warp_max(mx);
    if (threadIdx.x == 0) *out = mx;
  }
}

template <class ZC>
__global__ void k_diag_inv(int64_t N, const ZC *__restrict__ Z, const double *__restrict__ maxabs,
                           double2 *__restrict__ dinv) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double floor_abs = 1e-10 * (*maxabs);
  if (floor_abs == 0.0) floor_abs = 4.9406564584124654e-324;
  double2 z = to_d2(Z[i * N + i]);
  if (hypot(z.x, z.y) < floor_abs) z = make_double2(floor_abs, 0);
  dinv[i] = cdiv(make_double2(1, 0), z);
}

// ---------------------------------------------------------------------------
// LDL^T kernels; C is the storage and compute type (double2 or float2)
// ---------------------------------------------------------------------------
// Diagonal block: factor in shared memory, write L (strict lower) and D back,
// and write Linv = L11^-1 (unit lower, b x b, row-major NB stride).
//
// 256 threads as 16 x 16; thread (tx, ty) keeps entries (ty + 16p, tx + 16q),
// p, q in 0..3, of the block and of X = L^-1 in registers.  Elimination step k
// broadcasts column k of the block and row k of X through shared memory and
// applies both updates: L = L_0 L_1 ... with L_k = I + l_k e_k^T, so
// X = ... (I - l_1 e_1^T)(I - l_0 e_0^T), and row k of X is final once steps
// 0..k-1 have run.  One barrier pair per step covers both.
template <class C>
__device__ __forceinline__ void ldlt_diag_block(int64_t N, int64_t j, int b, C *__restrict__ F,
                                                C *__restrict__ Linv, unsigned *__restrict__ err, C *colk) {
  C *rowk = colk + NB;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  C a[4][4], x[4][4];
#pragma unroll
  for (int p = 0; p < 4; p++)
#pragma unroll
    for (int q = 0; q < 4; q++) {
      int i = ty + 16 * p, c = tx + 16 * q;
      a[p][q] = (i < b && c <= i) ? F[(j + i) * N + j + c] : czero<C>();
      x[p][q] = (i == c) ? cone<C>() : czero<C>();
    }
  for (int k = 0; k < b; k++) {
    const int kq = k >> 4;
    if (tx == (k & 15)) {
#pragma unroll
      for (int p = 0; p < 4; p++)
#pragma unroll
        for (int q = 0; q < 4; q++)
          if (q == kq) colk[ty + 16 * p] = a[p][q];
    }
    if (ty == (k & 15)) {
#pragma unroll
      for (int p = 0; p < 4; p++)
#pragma unroll
        for (int q = 0; q < 4; q++)
          if (p == kq) rowk[tx + 16 * q] = x[p][q];
    }
    __syncthreads();
    const C d = colk[k];
    const double ad = (double)cabsv(d);
    if (!(ad > 0.0) || !isfinite(ad)) {
      if (threadIdx.x == 0) atomicOr(err, 2u);
      return;  // uniform: every thread read the same pivot
    }
    const C inv_d = cdiv(cone<C>(), d);
    C l[4], xr[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      l[q] = cmul(colk[tx + 16 * q], inv_d);
      xr[q] = rowk[tx + 16 * q];
    }
    // warp-uniform skips: row blocks entirely at or above k, column blocks of
    // the block entirely left of k, and columns of X right of k (row k of X
    // is zero there) hold nothing to update
#pragma unroll
    for (int p = 0; p < 4; p++) {
      if (16 * p + 15 <= k) continue;
      const int i = ty + 16 * p;
      const C ci = colk[i];
      const C lik = cmul(ci, inv_d);
#pragma unroll
      for (int q = 0; q <= p; q++) {
        if (16 * q + 15 < k) continue;
        const int c = tx + 16 * q;
        if (c > k && c <= i) a[p][q] = csub(a[p][q], cmul(ci, l[q]));
        if (c == k && i > k) a[p][q] = lik;  // L entry of column k
      }
#pragma unroll
      for (int q = 0; q < 4; q++) {
        if (16 * q > k) continue;
        if (i > k) x[p][q] = csub(x[p][q], cmul(lik, xr[q]));
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int p = 0; p < 4; p++)
#pragma unroll
    for (int q = 0; q < 4; q++) {
      int i = ty + 16 * p, c = tx + 16 * q;
      if (i < b && c <= i) F[(j + i) * N + j + c] = a[p][q];
      Linv[i * NB + c] = x[p][q];
    }
}

// 1 / x for a positive normal float: the hardware approximation refined by
// one Newton-Raphson step, r <- r (2 - x r)
__device__ __forceinline__ float rcp_nr(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r * fmaf(-x, r, 2.f);
}
__device__ __forceinline__ float2 csel(bool p, float2 a, float2 b) { return make_float2(p ? a.x : b.x, p ? a.y : b.y); }

// Elimination of the 16 x 16 diagonal sub-block at s0 by one warp, all in
// registers: lane (ih = lane >> 4, c = lane & 15) holds rows i = ih + 2 m
// (m = 0..7) of column c.  The block is kept in full (both triangles: it is
// complex symmetric and every update keeps it so), which puts each value a
// pivot step needs -- the pivot, A[k][c] = A[c][k], X[k][c] and A[i][k] -- in
// a register whose index is known at compile time on a lane known per lane,
// so one shuffle fetches it; no shared memory, no warp barriers.  The updates
// are selects, not branches (the lane conditions differ within the warp).  On
// return the lower triangle holds L (strict) and D, X the unit-lower inverse.
// 1/d = conj(d) / |d|^2 with |d|^2 inverted by rcp_nr; a pivot whose |d|^2 is
// zero, non-finite or outside the FP32 normal range (|d| below ~1e-19 or above
// ~1e19) is a breakdown (false, uniform over the warp, decided after the 16
// steps).
__device__ __forceinline__ bool elim16_warp(float2 (*A)[65], float2 (*Xs)[17], int s0, int lane) {
  const unsigned FULL = 0xffffffffu;
  const int c = lane & 15, ih = lane >> 4;
  float2 a[8], x[8];
#pragma unroll
  for (int m = 0; m < 8; m++) {
    const int i = ih + 2 * m;
    a[m] = (c <= i) ? A[s0 + i][s0 + c] : A[s0 + c][s0 + i];
    x[m] = (i == c) ? make_float2(1.f, 0.f) : make_float2(0.f, 0.f);
  }
  bool ok = true;
#pragma unroll
  for (int k = 0; k < 16; k++) {
    const int kl = (k & 1) << 4, km = k >> 1;
    float2 d, akc, xk, aik[8];
    d.x = __shfl_sync(FULL, a[km].x, kl | k);
    d.y = __shfl_sync(FULL, a[km].y, kl | k);
    akc.x = __shfl_sync(FULL, a[km].x, kl | c);
    akc.y = __shfl_sync(FULL, a[km].y, kl | c);
    xk.x = __shfl_sync(FULL, x[km].x, kl | c);
    xk.y = __shfl_sync(FULL, x[km].y, kl | c);
#pragma unroll
    for (int m = 0; m < 8; m++) {
      aik[m].x = __shfl_sync(FULL, a[m].x, (ih << 4) | k);
      aik[m].y = __shfl_sync(FULL, a[m].y, (ih << 4) | k);
    }
    const float d2 = fmaf(d.x, d.x, d.y * d.y);
    ok = ok && (d2 >= 1.17549435e-38f) && (d2 <= 3.40282347e38f);
    const float rd = rcp_nr(d2);
    const float2 inv_d = make_float2(d.x * rd, -d.y * rd);
    const float2 lc = cmul(akc, inv_d);
#pragma unroll
    for (int m = 0; m < 8; m++) {
      const int i = ih + 2 * m;
      const bool below = i > k;
      const float2 lik = cmul(aik[m], inv_d);
      const float2 upd = csub(a[m], cmul(aik[m], lc));
      a[m] = csel(below && c > k, upd, csel(below && c == k, lik, a[m]));
      x[m] = csel(below, csub(x[m], cmul(lik, xk)), x[m]);
    }
  }
  if (!__all_sync(FULL, ok)) return false;
#pragma unroll
  for (int m = 0; m < 8; m++) {
    const int i = ih + 2 * m;
    if (c <= i) A[s0 + i][s0 + c] = a[m];
    Xs[i][c] = x[m];
  }
  return true;
}


// Blocked form of ldlt_diag_block for complex64 blocks (same results up to
// rounding): four 16-wide sub-panels; warp 0 eliminates the 16 x 16 diagonal
// sub-block in registers (elim16_warp, which also forms its unit-lower
// inverse), then the CTA computes the sub-panel below it (up to three rows
// per thread, accumulated together) and the trailing update (four columns per
// thread).  The 64 x 64 inverse is assembled from the four 16 x 16 inverses
// by recursive doubling (16-wide pairs, then the 32-wide halves), each phase
// a small product with several independent sums per thread.
// Rows and columns at or beyond b are padded with the identity (D = 1, L = 0).
constexpr size_t DIAG_BLOCKED_SMEM = sizeof(float2) * (2 * 64 * 65 + 64 * 17 + 4 * 16 * 17 + 16) + 16;

// The diagonal tile as the blocked factorisation expects it in shared memory:
// lower triangle of F at (j, j), zeros above, identity padding beyond b.
__device__ __forceinline__ void diag_tile_load(int64_t N, int64_t j, int b, const float2 *__restrict__ F,
                                               float2 (*A)[65]) {
  const int t = threadIdx.x;
  float2 v[16];
#pragma unroll
  for (int m = 0; m < 16; m++) {
    const int e = t + 256 * m, i = e >> 6, c = e & 63;
    v[m] = make_float2(0.f, 0.f);
    if (i < b && c < b) {
      if (c <= i) v[m] = __ldcg(F + (j + i) * N + j + c);
    } else if (i == c) {
      v[m] = make_float2(1.f, 0.f);
    }
  }
#pragma unroll
  for (int m = 0; m < 16; m++) {
    const int e = t + 256 * m;
    A[e >> 6][e & 63] = v[m];
  }
}

// The panel step's update of the next diagonal tile, applied to the tile in
// shared memory: A[r][c] -= sum_{k<K} W[j + r][woff + k] F[j + c][jcol + k]
// for c <= r < b (the same products and order as ldlt_tile_update).  The K
// chunks of 16 are staged in two buffers (the space of the inverse, unused
// until the end of the factorisation), the next chunk's loads in flight while
// the current one is multiplied.
__device__ __forceinline__ void diag_tile_update_smem(int64_t N, int64_t j, int b, int64_t jcol, int K,
                                                      const float2 *__restrict__ F, const float2 *__restrict__ W,
                                                      int wstride, int woff, float2 (*A)[65],
                                                      float2 (*St)[16][65]) {
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  float2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int jj = 0; jj < 4; jj++) acc[i][jj] = make_float2(0.f, 0.f);
  const int nch = (K + 15) / 16;
  float2 rw[4], rl[4];
  auto fetch = [&](int k0) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int e = threadIdx.x + 256 * q, kk = e & 15, rr = e >> 4;
      const bool ok = rr < b && k0 + kk < K;
      rw[q] = ok ? __ldcg(W + (j + rr) * wstride + woff + k0 + kk) : make_float2(0.f, 0.f);
      rl[q] = ok ? __ldcg(F + (j + rr) * N + jcol + k0 + kk) : make_float2(0.f, 0.f);
    }
  };
  auto stage = [&](int buf) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int e = threadIdx.x + 256 * q, kk = e & 15, rr = e >> 4;
      St[2 * buf][kk][rr] = rw[q];
      St[2 * buf + 1][kk][rr] = rl[q];
    }
  };
  fetch(0);
  stage(0);
  __syncthreads();
  for (int c = 0; c < nch; c++) {
    if (c + 1 < nch) fetch(16 * (c + 1));
    const int buf = c & 1;
#pragma unroll
    for (int kk = 0; kk < 16; kk++) {
      float2 a[4], l[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = St[2 * buf][kk][ty + 16 * i];
#pragma unroll
      for (int jj = 0; jj < 4; jj++) l[jj] = St[2 * buf + 1][kk][tx + 16 * jj];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int jj = 0; jj < 4; jj++) cfma(acc[i][jj], a[i], l[jj]);
    }
    if (c + 1 < nch) stage(buf ^ 1);
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int jj = 0; jj < 4; jj++) {
      const int r = ty + 16 * i, cc = tx + 16 * jj;
      if (r < b && cc <= r) A[r][cc] = csub(A[r][cc], acc[i][jj]);
    }
  __syncthreads();
}

// Phase 1 of the blocked factorisation: L and D of the diagonal tile (in
// shared memory, written back to F) and the unit-lower inverses Xd of its
// four 16 x 16 diagonal blocks.  loaded: the tile is already in shared memory
// (diag_tile_load, possibly updated by diag_tile_update_smem).  Returns false
// after a breakdown (uniform).
__device__ bool ldlt_diag_phase1(int64_t N, int64_t j, int b, float2 *__restrict__ F, unsigned *__restrict__ err,
                                 unsigned char *smem, bool loaded) {
  float2(*A)[65] = reinterpret_cast<float2(*)[65]>(smem);
  float2(*Wp)[17] = reinterpret_cast<float2(*)[17]>(smem + sizeof(float2) * 64 * 65);
  float2(*Xd)[16][17] = reinterpret_cast<float2(*)[16][17]>(smem + sizeof(float2) * (64 * 65 + 64 * 17));
  float2 *dinv = reinterpret_cast<float2 *>(smem + sizeof(float2) * (2 * 64 * 65 + 64 * 17 + 4 * 16 * 17));
  volatile int *bad = reinterpret_cast<volatile int *>(dinv + 16);
  const int t = threadIdx.x;  // 256 threads
  if (!loaded) {
    float2 v[16];
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int e = t + 256 * m, i = e >> 6, c = e & 63;
      v[m] = make_float2(0.f, 0.f);
      if (i < b && c < b) {
        if (c <= i) v[m] = F[(j + i) * N + j + c];
      } else if (i == c) {
        v[m] = make_float2(1.f, 0.f);
      }
    }
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int e = t + 256 * m;
      A[e >> 6][e & 63] = v[m];
    }
  }
  if (t == 0) *bad = 0;
  __syncthreads();
  for (int s = 0; s < 4; s++) {
    const int s0 = 16 * s;
    if (t < 32) {
      if (!elim16_warp(A, Xd[s], s0, t)) {  // uniform over the warp
        if (t == 0) {
          atomicOr(err, 2u);
          *bad = 1;
        }
      }
    }
    __syncthreads();
    if (*bad) return false;  // uniform
    if (s == 3) break;
    const int nr = 48 - s0;
    // 1 / D of the 16 pivots; sub-panel W = A21 X^T with up to three outputs
    // per thread accumulated together
    if (t < 16) {
      const float2 dd = A[s0 + t][s0 + t];
      const float rd = rcp_nr(fmaf(dd.x, dd.x, dd.y * dd.y));
      dinv[t] = make_float2(dd.x * rd, -dd.y * rd);
    }
    {
      float2 acc[3];
      int rr[3];
      const int c = t & 15;
#pragma unroll
      for (int u = 0; u < 3; u++) {
        acc[u] = make_float2(0.f, 0.f);
        rr[u] = s0 + 16 + (t >> 4) + 16 * u;
      }
#pragma unroll
      for (int k = 0; k < 16; k++) {
        if (k <= c) {
          const float2 xk = Xd[s][c][k];
#pragma unroll
          for (int u = 0; u < 3; u++)
            if (rr[u] < 64) cfma(acc[u], A[rr[u]][s0 + k], xk);
        }
      }
#pragma unroll
      for (int u = 0; u < 3; u++)
        if (rr[u] < 64) Wp[rr[u]][c] = acc[u];
    }
    __syncthreads();
    for (int e = t; e < nr * 16; e += blockDim.x) {
      const int r = s0 + 16 + (e >> 4), c = e & 15;
      A[r][s0 + c] = cmul(Wp[r][c], dinv[c]);
    }
    __syncthreads();
    // trailing update A22 -= W L21^T on the lower part: thread -> (row, 4 columns)
    {
      const int ncq = (nr + 3) / 4;  // column quads
      for (int e = t; e < nr * ncq; e += blockDim.x) {
        const int i = s0 + 16 + e / ncq, j0 = s0 + 16 + 4 * (e % ncq);
        if (j0 > i) continue;
        float2 acc[4] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
#pragma unroll
        for (int k = 0; k < 16; k++) {
          const float2 w = Wp[i][k];
#pragma unroll
          for (int q = 0; q < 4; q++) cfma(acc[q], w, A[min(j0 + q, 63)][s0 + k]);
        }
#pragma unroll
        for (int q = 0; q < 4; q++)
          if (j0 + q <= i) A[i][j0 + q] = csub(A[i][j0 + q], acc[q]);
      }
    }
    __syncthreads();
    }
  for (int e = t; e < 64 * 64; e += blockDim.x) {
    const int i = e >> 6, c = e & 63;
    if (i < b && c <= i) F[(j + i) * N + j + c] = A[i][c];
  }
  return true;
}

// Phase 2: the unit-lower inverse of the factored tile (L in shared memory)
// by recursive doubling from the four 16 x 16 inverses of phase 1, and its
// store to Linv.
__device__ void ldlt_diag_phase2(float2 *__restrict__ Linv, unsigned char *smem, bool skip_diag_blocks = false) {
  float2(*A)[65] = reinterpret_cast<float2(*)[65]>(smem);
  float2(*Wp)[17] = reinterpret_cast<float2(*)[17]>(smem + sizeof(float2) * 64 * 65);
  float2(*Xd)[16][17] = reinterpret_cast<float2(*)[16][17]>(smem + sizeof(float2) * (64 * 65 + 64 * 17));
  float2(*LI)[65] = reinterpret_cast<float2(*)[65]>(smem + sizeof(float2) * (64 * 65 + 64 * 17 + 4 * 16 * 17));
  const int t = threadIdx.x;
  // Linv by recursive doubling: 16-level pairs, then the 32-level block
  //   [[X0, 0], [-X1 L10 X0, X1]]
  for (int e = t; e < 64 * 64; e += blockDim.x) {
    const int i = e >> 6, c = e & 63;
    LI[i][c] = ((i >> 4) == (c >> 4)) ? Xd[i >> 4][i & 15][c & 15] : make_float2(0.f, 0.f);
  }
  // phase A: T_h = L[32h+16.., 32h..] Xd[2h] (two 16 x 16 products, 2 outputs per thread)
  {
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int e = t + 256 * u, h = e >> 8, r = (e >> 4) & 15, c = e & 15;
      float2 p0 = make_float2(0.f, 0.f), p1 = make_float2(0.f, 0.f);
#pragma unroll
      for (int k = 0; k < 16; k += 2) {
        cfma(p0, A[32 * h + 16 + r][32 * h + k], Xd[2 * h][k][c]);
        cfma(p1, A[32 * h + 16 + r][32 * h + k + 1], Xd[2 * h][k + 1][c]);
      }
      Wp[32 * h + r][c] = cadd(p0, p1);
    }
  }
  __syncthreads();
  // phase B: LI[32h+16+r][32h+c] = -Xd[2h+1] T_h
  {
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int e = t + 256 * u, h = e >> 8, r = (e >> 4) & 15, c = e & 15;
      float2 p0 = make_float2(0.f, 0.f), p1 = make_float2(0.f, 0.f);
#pragma unroll
      for (int k = 0; k < 16; k += 2) {
        if (k <= r) cfma(p0, Xd[2 * h + 1][r][k], Wp[32 * h + k][c]);
        if (k + 1 <= r) cfma(p1, Xd[2 * h + 1][r][k + 1], Wp[32 * h + k + 1][c]);
      }
      const float2 acc = cadd(p0, p1);
      LI[32 * h + 16 + r][32 * h + c] = make_float2(-acc.x, -acc.y);
    }
  }
  __syncthreads();
  // phase C: U = L[32.., 0..32) X_a (32 x 32, X_a lower: k >= c), 4 outputs
  // per thread; U goes to Wp as two 32 x 16 halves (Wp[r][c] for c < 16,
  // Wp[32 + r][c - 16] for c >= 16)
  {
    const int c = t & 31, r0 = t >> 5;  // rows r0, r0 + 8, r0 + 16, r0 + 24
    float2 p[4] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
#pragma unroll
    for (int k = 0; k < 32; k++) {
      if (k >= c) {
        const float2 x = LI[k][c];
#pragma unroll
        for (int q = 0; q < 4; q++) cfma(p[q], A[32 + r0 + 8 * q][k], x);
      }
    }
    __syncthreads();  // Wp of phase B is consumed
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int r = r0 + 8 * q;
      if (c < 16) Wp[r][c] = p[q];
      else Wp[32 + r][c - 16] = p[q];
    }
  }
  __syncthreads();
  // phase D: LI[32 + r][c] = -X_b U, X_b = LI[32.., 32..] lower (k <= r)
  {
    const int c = t & 31, r0 = t >> 5;
    float2 p[4] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
#pragma unroll
    for (int k = 0; k < 32; k++) {
      const float2 u = c < 16 ? Wp[k][c] : Wp[32 + k][c - 16];
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (k <= r0 + 8 * q) cfma(p[q], LI[32 + r0 + 8 * q][32 + k], u);
    }
#pragma unroll
    for (int q = 0; q < 4; q++) LI[32 + r0 + 8 * q][c] = make_float2(-p[q].x, -p[q].y);
  }
  __syncthreads();
  // (skip_diag_blocks: the 16 x 16 diagonal blocks were stored already)
  for (int e = t; e < 64 * 64; e += blockDim.x)
    if (!skip_diag_blocks || (e >> 10) != ((e & 63) >> 4)) Linv[e] = LI[e >> 6][e & 63];
  __syncthreads();
}

// Blocked form of ldlt_diag_block for complex64 blocks: phase 1 (with the
// 16 x 16 inverses), the store of L and D, phase 2.
__device__ void ldlt_diag_blocked(int64_t N, int64_t j, int b, float2 *__restrict__ F, float2 *__restrict__ Linv,
                                  unsigned *__restrict__ err, unsigned char *smem, bool loaded = false) {
  if (!ldlt_diag_phase1(N, j, b, F, err, smem, loaded)) return;
  ldlt_diag_phase2(Linv, smem);
}
template <class C>
__global__ void __launch_bounds__(256) k_ldlt_diag(int64_t N, int64_t j, int b, C *__restrict__ F,
                                                   C *__restrict__ Linv, unsigned *__restrict__ err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if constexpr (std::is_same<C, float2>::value)
    ldlt_diag_blocked(N, j, b, F, Linv, err, smem_raw);
  else
    ldlt_diag_block<C>(N, j, b, F, Linv, err, reinterpret_cast<C *>(smem_raw));
}

// Panel: W = A21 Linv^T (row r: W[r][c] = sum_{k<=c} A21[r][k] Linv[c][k]),
// then L21 = W D^-1, for the 64 rows from r0.  Reads go through L2 (the
// fused step kernel reads blocks written by another CTA of the same launch).
// a_in_smem: the A21 tile is already in As (ldlt_strip_update_smem)
template <class C>
__device__ __forceinline__ void ldlt_panel_rows(int64_t N, int64_t j, int b, int64_t r0, C *__restrict__ F,
                                                const C *__restrict__ Linv, C *__restrict__ W, int wstride,
                                                int woff, unsigned char *smem_raw, bool a_in_smem = false) {
  C(*As)[NB + 1] = reinterpret_cast<C(*)[NB + 1]>(smem_raw);
  C(*Li)[NB + 1] = reinterpret_cast<C(*)[NB + 1]>(smem_raw + sizeof(C) * NB * (NB + 1));
  C *dg = reinterpret_cast<C *>(smem_raw + 2 * sizeof(C) * NB * (NB + 1));
  if (a_in_smem) {
    C vl[16];
#pragma unroll
    for (int m = 0; m < 16; m++) vl[m] = __ldcg(Linv + threadIdx.x + 256 * m);
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int e = threadIdx.x + 256 * m;
      Li[e / NB][e % NB] = vl[m];
    }
  } else {
    // 256 threads: all 32 loads of a thread in flight before the shared stores
    C va[16], vl[16];
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int e = threadIdx.x + 256 * m, rr = e / NB, k = e % NB;
      const int64_t r = r0 + rr;
      va[m] = (r < N && k < b) ? __ldcg(F + r * N + j + k) : czero<C>();
      vl[m] = __ldcg(Linv + rr * NB + k);
    }
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int e = threadIdx.x + 256 * m;
      As[e / NB][e % NB] = va[m];
      Li[e / NB][e % NB] = vl[m];
    }
  }
  if (threadIdx.x < b) dg[threadIdx.x] = __ldcg(F + (j + threadIdx.x) * N + j + threadIdx.x);
  __syncthreads();
  // thread (c, rq) owns column c of rows rq, rq + 4, ..., rq + 60: sixteen
  // independent accumulators per Linv entry
  const int c = threadIdx.x & 63, rq = threadIdx.x >> 6;
  if (c >= b) return;
  C acc[16];
#pragma unroll
  for (int t = 0; t < 16; t++) acc[t] = czero<C>();
  for (int k = 0; k <= c; k++) {
    const C lk = Li[c][k];
#pragma unroll
    for (int t = 0; t < 16; t++) cfma(acc[t], As[rq + 4 * t][k], lk);
  }
  const C inv = cdiv(cone<C>(), dg[c]);
#pragma unroll
  for (int t = 0; t < 16; t++) {
    const int64_t r = r0 + rq + 4 * t;
    if (r < N) {
      W[r * wstride + woff + c] = acc[t];
      F[r * N + j + c] = cmul(acc[t], inv);
    }
  }
}

template <class C>
__global__ void __launch_bounds__(256) k_ldlt_panel(int64_t N, int64_t j, int b, C *__restrict__ F,
                                                    const C *__restrict__ Linv, C *__restrict__ W, int wstride,
                                                    int woff) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ldlt_panel_rows<C>(N, j, b, j + b + (int64_t)blockIdx.x * NB, F, Linv, W, wstride, woff, smem_raw);
}

// Panel rows of the fused step by blocked forward substitution, W L11^T =
// A21 in four 16-column blocks: T_J = A21_J - sum_{K<J} W_K L_JK^T, then
// W_J = T_J X_J^T with X_J the inverse of L_JJ (the diagonal 16 x 16 blocks
// of the tile's inverse, published with L and D before the rest of the
// inverse exists).  A21 is already in As (ldlt_strip_update_smem); T and W
// overwrite it in place.  L21 = W D^-1 to F, W to the panel buffer.
__device__ __forceinline__ void ldlt_panel_rows_blk(int64_t N, int64_t j, int b, int64_t r0,
                                                    float2 *__restrict__ F, const float2 *__restrict__ Linv,
                                                    float2 *__restrict__ W, int wstride, int woff,
                                                    unsigned char *smem_raw) {
  float2(*As)[NB + 1] = reinterpret_cast<float2(*)[NB + 1]>(smem_raw);
  float2(*Lb)[NB + 1] = reinterpret_cast<float2(*)[NB + 1]>(smem_raw + sizeof(float2) * NB * (NB + 1));
  float2 *dinv = reinterpret_cast<float2 *>(smem_raw + 2 * sizeof(float2) * NB * (NB + 1));
  float2(*X)[16][17] = reinterpret_cast<float2(*)[16][17]>(smem_raw + 2 * sizeof(float2) * NB * (NB + 1) +
                                                          sizeof(float2) * NB);
  {
    float2 v[16], xv[4];
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int e = threadIdx.x + 256 * m, c = e >> 6, k = e & 63;
      v[m] = (c < b && k <= c) ? __ldcg(F + (j + c) * N + j + k) : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int e = threadIdx.x + 256 * q, J = e >> 8, i = (e >> 4) & 15, c = e & 15;
      xv[q] = __ldcg(Linv + (16 * J + i) * NB + 16 * J + c);
    }
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int e = threadIdx.x + 256 * m;
      Lb[e >> 6][e & 63] = v[m];
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int e = threadIdx.x + 256 * q;
      X[e >> 8][(e >> 4) & 15][e & 15] = xv[q];
    }
  }
  __syncthreads();
  if (threadIdx.x < b) dinv[threadIdx.x] = cdiv(make_float2(1.f, 0.f), Lb[threadIdx.x][threadIdx.x]);
  const int c = threadIdx.x & 15, rq = threadIdx.x >> 4;  // rows rq + 16 q
  for (int J = 0; J < 4; J++) {
    if (16 * J >= b) break;  // uniform
    float2 tq[4];
#pragma unroll
    for (int q = 0; q < 4; q++) tq[q] = As[rq + 16 * q][16 * J + c];
    for (int k = 0; k < 16 * J; k++) {
      const float2 l = Lb[16 * J + c][k];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const float2 w = As[rq + 16 * q][k];
        tq[q].x -= w.x * l.x - w.y * l.y;
        tq[q].y -= w.x * l.y + w.y * l.x;
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; q++) As[rq + 16 * q][16 * J + c] = tq[q];
    __syncthreads();
    float2 wq[4] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
#pragma unroll
    for (int k = 0; k < 16; k++) {
      if (k <= c) {
        const float2 x = X[J][c][k];
#pragma unroll
        for (int q = 0; q < 4; q++) cfma(wq[q], As[rq + 16 * q][16 * J + k], x);
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; q++) As[rq + 16 * q][16 * J + c] = wq[q];
    __syncthreads();
  }
  for (int e = threadIdx.x; e < 64 * 64; e += 256) {
    const int r = e >> 6, cc = e & 63;
    const int64_t gr = r0 + r;
    if (gr < N && cc < b) {
      const float2 w = As[r][cc];
      W[gr * wstride + woff + cc] = w;
      F[gr * N + j + cc] = cmul(w, dinv[cc]);
    }
  }
}

// F[r][c] -= sum_{k<K} W[r][woff+k] F[c][jcol+k] on the 64 x 64 tile at
// (r0, c0), c < c_hi, r >= c, r < N (SIMT; Ws / Ls: 2 x 16 x 65 staging)
template <class C>
__device__ __forceinline__ void ldlt_tile_update(int64_t N, int64_t r0, int64_t c0, int64_t c_hi, int64_t jcol,
                                                 int K, C *__restrict__ F, const C *__restrict__ W, int wstride,
                                                 int woff, C (*Ws)[65], C (*Ls)[65]) {
  int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  C acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int jj = 0; jj < 4; jj++) acc[i][jj] = czero<C>();
  for (int k0 = 0; k0 < K; k0 += 16) {
    for (int e = threadIdx.x; e < 16 * 64; e += 256) {
      int kk = e & 15, rr = e >> 4;
      int64_t r = r0 + rr, cc = c0 + rr;
      bool kin = k0 + kk < K;
      Ws[kk][rr] = (r < N && kin) ? W[r * wstride + woff + k0 + kk] : czero<C>();
      Ls[kk][rr] = (cc < c_hi && kin) ? F[cc * N + jcol + k0 + kk] : czero<C>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; kk++) {
      C a[4], l[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = Ws[kk][ty + 16 * i];
#pragma unroll
      for (int jj = 0; jj < 4; jj++) l[jj] = Ls[kk][tx + 16 * jj];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int jj = 0; jj < 4; jj++) cfma(acc[i][jj], a[i], l[jj]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int jj = 0; jj < 4; jj++) {
      int64_t r = r0 + ty + 16 * i, cc = c0 + tx + 16 * jj;
      if (r < N && cc < c_hi && cc <= r) {
        C *p = F + r * N + cc;
        *p = csub(*p, acc[i][jj]);
      }
    }
}

// The panel step's strip update of a column-0 tile (rows r0.., the next
// panel's columns c0.. = its diagonal block's), kept in shared memory as the
// A21 tile of the panel rows that follow (As: its first b columns, zeros
// beyond): the same products as ldlt_tile_update, without the round trip
// through F.  Ws / Ls staging past the panel's As / Li / dg space.
template <class C>
__device__ __forceinline__ void ldlt_strip_update_smem(int64_t N, int64_t r0, int64_t c0, int b, int64_t jcol,
                                                       int K, const C *__restrict__ F, const C *__restrict__ W,
                                                       int wstride, int woff, unsigned char *smem_raw) {
  C(*As)[NB + 1] = reinterpret_cast<C(*)[NB + 1]>(smem_raw);
  C(*Ws)[65] = reinterpret_cast<C(*)[65]>(smem_raw + 2 * sizeof(C) * NB * (NB + 1) + sizeof(C) * NB);
  C(*Ls)[65] = reinterpret_cast<C(*)[65]>(smem_raw + 2 * sizeof(C) * NB * (NB + 1) + sizeof(C) * NB +
                                          sizeof(C) * 16 * 65);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  C acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int jj = 0; jj < 4; jj++) acc[i][jj] = czero<C>();
  for (int k0 = 0; k0 < K; k0 += 16) {
    for (int e = threadIdx.x; e < 16 * 64; e += 256) {
      int kk = e & 15, rr = e >> 4;
      int64_t r = r0 + rr;
      bool kin = k0 + kk < K;
      Ws[kk][rr] = (r < N && kin) ? __ldcg(W + r * wstride + woff + k0 + kk) : czero<C>();
      Ls[kk][rr] = (rr < b && kin) ? __ldcg(F + (c0 + rr) * N + jcol + k0 + kk) : czero<C>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; kk++) {
      C a[4], l[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = Ws[kk][ty + 16 * i];
#pragma unroll
      for (int jj = 0; jj < 4; jj++) l[jj] = Ls[kk][tx + 16 * jj];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int jj = 0; jj < 4; jj++) cfma(acc[i][jj], a[i], l[jj]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int jj = 0; jj < 4; jj++) {
      const int rr = ty + 16 * i, k = tx + 16 * jj;
      const int64_t r = r0 + rr;
      As[rr][k] = (r < N && k < b) ? csub(__ldcg(F + r * N + c0 + k), acc[i][jj]) : czero<C>();
    }
}

// Trailing / strip update on tiles (grid.x row tiles, grid.y column tiles from
// r_lo; tiles entirely above the diagonal exit at once).
//
// diag_b > 0: the CTA of tile (0, 0) -- the diagonal block at r_lo, which is
// the next panel's -- factors that block right after updating it
// (ldlt_diag_block, Linv_next), while the other CTAs finish the strip.
template <class C>
__global__ void __launch_bounds__(256) k_ldlt_update(int64_t N, int64_t r_lo, int64_t c_hi, int64_t jcol, int K,
                                                     C *__restrict__ F, const C *__restrict__ W, int wstride,
                                                     int woff, int diag_b, C *__restrict__ Linv_next,
                                                     unsigned *__restrict__ err) {
  __shared__ C Ws[16][65];
  __shared__ C Ls[16][65];
  const int64_t r0 = r_lo + (int64_t)blockIdx.x * 64, c0 = r_lo + (int64_t)blockIdx.y * 64;
  if (r0 >= N || c0 >= c_hi || c0 > r0 + 63) return;
  ldlt_tile_update<C>(N, r0, c0, c_hi, jcol, K, F, W, wstride, woff, Ws, Ls);
  if (diag_b > 0 && blockIdx.x == 0 && blockIdx.y == 0) {
    __syncthreads();  // the tile's writes are visible to the whole CTA
    ldlt_diag_block<C>(N, r_lo, diag_b, F, Linv_next, err, &Ws[0][0]);
  }
}

// One panel step inside a 256-wide middle panel, fused: strip update of the
// columns [r_lo, c_hi) by the panel at jcol; the CTA holding ticket 0 updates
// the next diagonal block (tile (0, 0)), factors it and publishes its inverse
// (sync[1]); every other CTA of column tile 0 then runs the next panel on its
// own rows (W at woff_next, L21 = W D^-1).  Tickets are drawn in launch order,
// so the CTA that the others wait for is already running; the wait is bounded
// (error bit 4 on expiry).
template <class C>
__global__ void __launch_bounds__(256) k_ldlt_step(int64_t N, int64_t r_lo, int64_t c_hi, int64_t jcol, int K,
                                                   C *__restrict__ F, C *__restrict__ W, int wstride, int woff,
                                                   int woff_next, int nb_next, C *__restrict__ Linv_next,
                                                   unsigned *__restrict__ sync, unsigned *__restrict__ err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ unsigned s_ticket;
  __shared__ int s_ok;
  if (threadIdx.x == 0) s_ticket = atomicAdd(&sync[0], 1u);
  __syncthreads();
  const unsigned t = s_ticket;
  const int nct = (int)((c_hi - r_lo + 63) / 64);
  const int64_t rt = t / nct;
  const int ct = (int)(t % nct);
  const int64_t r0 = r_lo + rt * 64, c0 = r_lo + (int64_t)ct * 64;
  if (r0 >= N || c0 > r0 + 63) return;
  C(*Ws)[65] = reinterpret_cast<C(*)[65]>(smem_raw);
  C(*Ls)[65] = reinterpret_cast<C(*)[65]>(smem_raw + sizeof(C) * 16 * 65);
  if (t == 0) {
    // the next diagonal tile: loaded once, updated and factored in shared
    // memory (complex64); the update's K chunks are staged in the space of
    // the tile's inverse
    if constexpr (std::is_same<C, float2>::value) {
      float2(*A)[65] = reinterpret_cast<float2(*)[65]>(smem_raw);
      float2(*St)[16][65] =
          reinterpret_cast<float2(*)[16][65]>(smem_raw + sizeof(float2) * (64 * 65 + 64 * 17 + 4 * 16 * 17));
      diag_tile_load(N, r_lo, nb_next, F, A);
      diag_tile_update_smem(N, r_lo, nb_next, jcol, K, F, W, wstride, woff, A, St);
      // L, D and the 16 x 16 diagonal blocks of the inverse are published
      // first (the panel rows need only them); the rest of the tile's
      // inverse, for the solves, is formed while the panel rows run
      const bool ok = ldlt_diag_phase1(N, r_lo, nb_next, F, err, smem_raw, true);
      if (ok) {
        float2(*Xd)[16][17] = reinterpret_cast<float2(*)[16][17]>(smem_raw + sizeof(float2) * (64 * 65 + 64 * 17));
        for (int e = threadIdx.x; e < 4 * 256; e += 256) {
          const int s = e >> 8, i = (e >> 4) & 15, c = e & 15;
          Linv_next[(16 * s + i) * NB + 16 * s + c] = Xd[s][i][c];
        }
      }
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) atomicExch(&sync[1], 1u);
      if (ok) ldlt_diag_phase2(Linv_next, smem_raw, true);
    } else {
      ldlt_tile_update<C>(N, r0, c0, c_hi, jcol, K, F, W, wstride, woff, Ws, Ls);
      __syncthreads();
      ldlt_diag_block<C>(N, r_lo, nb_next, F, Linv_next, err, reinterpret_cast<C *>(smem_raw));
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) atomicExch(&sync[1], 1u);
    }
    return;
  }
  if (ct != 0) {
    ldlt_tile_update<C>(N, r0, c0, c_hi, jcol, K, F, W, wstride, woff, Ws, Ls);
    return;
  }
  // column 0: the strip tile is the next panel's A21 tile; it stays in
  // shared memory for the panel rows after the diagonal block is published
  ldlt_strip_update_smem<C>(N, r0, c0, nb_next, jcol, K, F, W, wstride, woff, smem_raw);
  if (threadIdx.x == 0) {
    long long it = 0;
    int ok = 1;
    while (*((volatile unsigned *)&sync[1]) == 0u) {
      if (++it > SPIN_LIMIT) {
        atomicOr(err, 4u);
        ok = 0;
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  if (!s_ok) return;
  if constexpr (std::is_same<C, float2>::value)
    ldlt_panel_rows_blk(N, r_lo, nb_next, r0, F, Linv_next, W, wstride, woff_next, smem_raw);
  else
    ldlt_panel_rows<C>(N, r_lo, nb_next, r0, F, Linv_next, W, wstride, woff_next, smem_raw, true);
}

// The first 64-wide block of a middle panel (complex64), one launch: the
// CTA holding ticket 0 factors the diagonal tile at j (phase 1), publishes
// L, D and the 16 x 16 inverse blocks, then forms the rest of the inverse
// (phase 2); every other CTA loads its 64 rows of the block column, waits for
// the publication (bounded, error bit 4 on expiry) and runs its panel rows
// by blocked forward substitution.  Replaces k_ldlt_diag + k_ldlt_panel.
__global__ void __launch_bounds__(256) k_ldlt_first(int64_t N, int64_t j, int b, float2 *__restrict__ F,
                                                    float2 *__restrict__ Linv, float2 *__restrict__ W, int wstride,
                                                    int woff, unsigned *__restrict__ sync,
                                                    unsigned *__restrict__ err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ unsigned s_ticket;
  __shared__ int s_ok;
  if (threadIdx.x == 0) s_ticket = atomicAdd(&sync[0], 1u);
  __syncthreads();
  const unsigned t = s_ticket;
  if (t == 0) {
    const bool ok = ldlt_diag_phase1(N, j, b, F, err, smem_raw, false);
    if (ok) {
      float2(*Xd)[16][17] = reinterpret_cast<float2(*)[16][17]>(smem_raw + sizeof(float2) * (64 * 65 + 64 * 17));
      for (int e = threadIdx.x; e < 4 * 256; e += 256) {
        const int s = e >> 8, i = (e >> 4) & 15, c = e & 15;
        Linv[(16 * s + i) * NB + 16 * s + c] = Xd[s][i][c];
      }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicExch(&sync[1], 1u);
    if (ok) ldlt_diag_phase2(Linv, smem_raw, true);
    return;
  }
  const int64_t r0 = j + b + (int64_t)(t - 1) * NB;
  if (r0 >= N) return;
  {
    float2(*As)[NB + 1] = reinterpret_cast<float2(*)[NB + 1]>(smem_raw);
    float2 va[16];
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int e = threadIdx.x + 256 * m, rr = e >> 6, k = e & 63;
      const int64_t r = r0 + rr;
      va[m] = (r < N && k < b) ? __ldcg(F + r * N + j + k) : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int e = threadIdx.x + 256 * m;
      As[e >> 6][e & 63] = va[m];
    }
  }
  if (threadIdx.x == 0) {
    long long it = 0;
    int ok = 1;
    while (*((volatile unsigned *)&sync[1]) == 0u) {
      if (++it > SPIN_LIMIT) {
        atomicOr(err, 4u);
        ok = 0;
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  if (!s_ok) return;
  ldlt_panel_rows_blk(N, j, b, r0, F, Linv, W, wstride, woff, smem_raw);
}

// ---------------------------------------------------------------------------
// ticket-ordered triangular solves (one right-hand side per grid.y)
// ---------------------------------------------------------------------------
// wait until flag[cb] is set; return how many consecutive flags from cb on are
// set (>= 1), or 0 when the wait expired (error bit 4 recorded)
__device__ int wait_flags(const volatile unsigned *fl, int cb, int limit, unsigned *err, long long spin_limit) {
  long long it = 0;
  while (fl[cb] == 0u) {
    if (++it > spin_limit) {
      atomicOr(err, 4u);
      return 0;
    }
    if (*((volatile unsigned *)err) & 4u) return 0;
    __nanosleep(64);
  }
  int r = cb + 1;
  while (r < limit && fl[r] != 0u) r++;
  return r - cb;
}

// 64 x 64 matrix (shared memory, row stride NB) times a 64-vector (shared
// memory) with four threads per output: thread (o = tid >> 2, part = tid & 3)
// sums 16 terms, two shuffles combine the parts.  TR: the matrix is read
// transposed (output o takes column o).  Every thread returns the sum of its
// output.
template <class FC, bool TR>
__device__ __forceinline__ double2 gemv64_quad(const FC *__restrict__ M, const double2 *__restrict__ v) {
  const int o = threadIdx.x >> 2, part = threadIdx.x & 3;
  double2 a = make_double2(0, 0), b = make_double2(0, 0);
#pragma unroll
  for (int k = 0; k < 16; k += 2) {
    const int c0 = part * 16 + k, c1 = c0 + 1;
    cfma(a, to_d2(TR ? M[c0 * NB + o] : M[o * NB + c0]), v[c0]);
    cfma(b, to_d2(TR ? M[c1 * NB + o] : M[o * NB + c1]), v[c1]);
  }
  a = cadd(a, b);
  a.x += __shfl_xor_sync(0xffffffffu, a.x, 1);
  a.y += __shfl_xor_sync(0xffffffffu, a.y, 1);
  a.x += __shfl_xor_sync(0xffffffffu, a.x, 2);
  a.y += __shfl_xor_sync(0xffffffffu, a.y, 2);
  return a;
}

// L y = x (x overwritten), L unit lower.  256 threads = 4 row groups x 64
// columns; while earlier block rows are streamed each thread accumulates its
// 16 rows across all solved block rows in registers, and those partial sums
// are reduced before the last wait.  The L block of the last dependency
// (block row t-1) and the inverse diagonal block are staged in shared memory
// before any wait, so the critical path after the last flag is one L2 read of
// y_{t-1} into shared memory and two 64 x 64 products on chip (four threads
// per row, two shuffles each).
template <class FC>
__global__ void __launch_bounds__(256) k_trsv_fwd(int64_t N, const FC *__restrict__ F, const FC *__restrict__ Linv,
                                                  double2 *x, unsigned *flags, unsigned *tickets, unsigned *err,
                                                  long long spin_limit) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  FC *Lp = reinterpret_cast<FC *>(smem_raw);
  FC *Li = Lp + NB * NB;
  __shared__ double2 acc[NB];
  __shared__ double2 ys[NB];
  __shared__ double2 part[2][NB];
  __shared__ int s_t, s_n;
  const int nblk = (int)((N + NB - 1) / NB);
  const int rhs = blockIdx.y;
  double2 *xr = x + (int64_t)rhs * N;
  unsigned *fl = flags + (int64_t)rhs * nblk;
  if (threadIdx.x == 0) s_t = (int)atomicAdd(tickets + rhs, 1u);
  __syncthreads();
  const int t = s_t;
  const int64_t r0 = (int64_t)t * NB;
  const int bs = (int)(N - r0 < NB ? N - r0 : NB);
  const int col = threadIdx.x & 63, rg = threadIdx.x >> 6, half = (threadIdx.x >> 5) & 1;
  // stage Linv_tt and, for t > 0, L[r0.., (t-1)*NB..]
  const FC *Lit = Linv + (int64_t)t * NB * NB;
  for (int e = threadIdx.x; e < NB * NB; e += 256) {
    Li[e] = Lit[e];
    int row = e >> 6, cc = e & 63;
    if (t > 0) Lp[e] = row < bs ? F[(r0 + row) * N + (int64_t)(t - 1) * NB + cc] : FC{};
  }
  double2 p[16];
#pragma unroll
  for (int i = 0; i < 16; i++) p[i] = make_double2(0, 0);
  int cb = 0;
  while (cb < t - 1) {
    if (threadIdx.x == 0) s_n = wait_flags(fl, cb, t - 1, err, spin_limit);
    __syncthreads();
    const int n = s_n;
    __syncthreads();
    if (n == 0) return;
    __threadfence();
    for (int q = cb; q < cb + n; q++) {
      const int64_t c0 = (int64_t)q * NB;
      const double2 yv = __ldcg(xr + c0 + col);
#pragma unroll
      for (int i = 0; i < 16; i++) {
        int row = rg + 4 * i;
        if (row < bs) cfma(p[i], to_d2(F[(r0 + row) * N + c0 + col]), yv);
      }
    }
    cb += n;
  }
  // acc = x_t - (streamed block rows), before the last wait
  if (threadIdx.x < NB) acc[threadIdx.x] = threadIdx.x < bs ? xr[r0 + threadIdx.x] : make_double2(0, 0);
#pragma unroll
  for (int i = 0; i < 16; i++) {
    double2 v = warp_sum2(p[i]);
    if ((threadIdx.x & 31) == 0) part[half][rg + 4 * i] = v;
  }
  __syncthreads();
  if (threadIdx.x < NB) acc[threadIdx.x] = csub(acc[threadIdx.x], cadd(part[0][threadIdx.x], part[1][threadIdx.x]));
  if (t > 0) {
    if (threadIdx.x == 0) s_n = wait_flags(fl, t - 1, t, err, spin_limit);
    __syncthreads();
    if (s_n == 0) return;
    __threadfence();
    if (threadIdx.x < NB) ys[threadIdx.x] = __ldcg(xr + (int64_t)(t - 1) * NB + threadIdx.x);
    __syncthreads();
    const double2 v = gemv64_quad<FC, false>(Lp, ys);
    if ((threadIdx.x & 3) == 0) acc[threadIdx.x >> 2] = csub(acc[threadIdx.x >> 2], v);
  }
  __syncthreads();
  // y_t = Linv_tt acc
  const double2 y = gemv64_quad<FC, false>(Li, acc);
  if ((threadIdx.x & 3) == 0 && (threadIdx.x >> 2) < bs) xr[r0 + (threadIdx.x >> 2)] = y;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) atomicExch(fl + t, 1u);
}

// L^T x = z (x overwritten), block rows bottom-up; flags indexed by ticket
// (ticket 0 = last block row).  Thread (rq, col) handles column col of the
// solved block rows' L entries, rows rq + 4i.  The L block of the last
// dependency (block row t+1) and Linv_tt are staged before any wait.
template <class FC>
__global__ void __launch_bounds__(256) k_trsv_bwd(int64_t N, const FC *__restrict__ F, const FC *__restrict__ Linv,
                                                  double2 *x, unsigned *flags, unsigned *tickets, unsigned *err,
                                                  long long spin_limit) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  FC *Lp = reinterpret_cast<FC *>(smem_raw);
  FC *Li = Lp + NB * NB;
  __shared__ double2 acc[NB];
  __shared__ double2 part[4][NB];
  __shared__ int s_t, s_n;
  const int nblk = (int)((N + NB - 1) / NB);
  const int rhs = blockIdx.y;
  double2 *xr = x + (int64_t)rhs * N;
  unsigned *fl = flags + (int64_t)rhs * nblk;
  if (threadIdx.x == 0) s_t = (int)atomicAdd(tickets + rhs, 1u);
  __syncthreads();
  const int tk = s_t;
  const int t = nblk - 1 - tk;
  const int64_t r0 = (int64_t)t * NB;
  const int bs = (int)(N - r0 < NB ? N - r0 : NB);
  const int col = threadIdx.x & 63, rq = threadIdx.x >> 6;
  const FC *Lit = Linv + (int64_t)t * NB * NB;
  const int64_t cl0 = (int64_t)(t + 1) * NB;  // last dependency block row
  const int cls = tk > 0 ? (int)(N - cl0 < NB ? N - cl0 : NB) : 0;
  for (int e = threadIdx.x; e < NB * NB; e += 256) {
    Li[e] = Lit[e];
    int r = e >> 6, cc = e & 63;
    if (tk > 0) Lp[e] = (r < cls && cc < bs) ? F[(cl0 + r) * N + r0 + cc] : FC{};
  }
  double2 s = make_double2(0, 0);
  int q0 = 0;
  while (q0 < tk - 1) {
    if (threadIdx.x == 0) s_n = wait_flags(fl, q0, tk - 1, err, spin_limit);
    __syncthreads();
    const int n = s_n;
    __syncthreads();
    if (n == 0) return;
    __threadfence();
    for (int q = q0; q < q0 + n; q++) {
      const int cb = nblk - 1 - q;
      const int64_t c0 = (int64_t)cb * NB;
      const int cbs = (int)(N - c0 < NB ? N - c0 : NB);
      if (col < bs)
        for (int r = rq; r < cbs; r += 4) cfma(s, to_d2(F[(c0 + r) * N + r0 + col]), __ldcg(xr + c0 + r));
    }
    q0 += n;
  }
  if (tk > 0) {
    if (threadIdx.x == 0) s_n = wait_flags(fl, tk - 1, tk, err, spin_limit);
    __syncthreads();
    if (s_n == 0) return;
    __threadfence();
    for (int r = rq; r < cls; r += 4) cfma(s, to_d2(Lp[r * NB + col]), __ldcg(xr + cl0 + r));
  }
  part[rq][col] = s;
  if (threadIdx.x < NB) acc[threadIdx.x] = threadIdx.x < bs ? xr[r0 + threadIdx.x] : make_double2(0, 0);
  __syncthreads();
  if (threadIdx.x < NB)
    acc[threadIdx.x] = csub(acc[threadIdx.x], cadd(cadd(part[0][threadIdx.x], part[1][threadIdx.x]),
                                                   cadd(part[2][threadIdx.x], part[3][threadIdx.x])));
  __syncthreads();
  // x_t = Linv_tt^T acc: x[c] = sum_r Linv[r][c] acc[r]
  s = make_double2(0, 0);
  for (int r = rq; r < NB; r += 4) cfma(s, to_d2(Li[r * NB + col]), acc[r]);
  part[rq][col] = s;
  __syncthreads();
  if (threadIdx.x < bs)
    xr[r0 + threadIdx.x] = cadd(cadd(part[0][threadIdx.x], part[1][threadIdx.x]),
                                cadd(part[2][threadIdx.x], part[3][threadIdx.x]));
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) atomicExch(fl + tk, 1u);
}

template <class FC>
__global__ void k_scale_by_dinv(int64_t N, int64_t R, const FC *__restrict__ F, double2 *__restrict__ x) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N * R) return;
  int64_t n = i % N;
  x[i] = cdiv(x[i], to_d2(F[n * N + n]));
}

__global__ void k_scale_vec(int64_t N, int64_t R, const double2 *__restrict__ d, double2 *__restrict__ x) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N * R) return;
  x[i] = cmul(x[i], d[i % N]);
}

template <class C> size_t diag_smem() {
  return std::is_same<C, float2>::value ? DIAG_BLOCKED_SMEM : sizeof(C) * 2 * NB;
}

template <class C> void set_smem_attrs() {
  static bool done = false;
  if (done) return;
  size_t panel = sizeof(C) * (2 * NB * (NB + 1) + NB);
  DMB_CUDA(cudaFuncSetAttribute(k_ldlt_panel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)panel));
  DMB_CUDA(cudaFuncSetAttribute(k_ldlt_diag<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)diag_smem<C>()));
  DMB_CUDA(cudaFuncSetAttribute(k_ldlt_step<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)std::max(panel, diag_smem<C>())));
  if constexpr (std::is_same<C, float2>::value)
    DMB_CUDA(cudaFuncSetAttribute(k_ldlt_first, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)std::max(panel, diag_smem<C>())));
  DMB_CUDA(cudaFuncSetAttribute(k_trsv_fwd<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(2 * sizeof(C) * NB * NB)));
  DMB_CUDA(cudaFuncSetAttribute(k_trsv_bwd<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(2 * sizeof(C) * NB * NB)));
  done = true;
}

// Three-level right-looking LDL^T.  Block columns of NBW = 1024 are factored
// as 256-wide middle panels, each made of four 64-wide panels (diagonal block,
// panel, SIMT strip updates inside the 256 columns).  After each middle panel
// the rest of the 1024-wide block column receives one K = 256 update, and after
// the block column the whole trailing matrix receives one K = 1024 update --
// both on the tensor cores for complex64 factors.
//
// Lookahead (details at update_block_column / update_trailing): the next
// panel's latency-bound diagonal/panel/strip kernels run on the main stream
// while the rest of each update streams through the tensor cores on two side
// streams, always on columns disjoint from the main stream's.
constexpr int NBO = 256;
constexpr int NBW = 1024;

template <class C> void ldlt_factor(dmb_ctx *c, C *F) {
  c->f_version++;  // F changes from here on: packed copies are stale
  const int64_t N = c->n;
  set_smem_attrs<C>();
  const int nblk = (int)((N + NB - 1) / NB);
  c->d_W.ensure(sizeof(C) * N * NBW * 2);
  c->d_dinv.ensure(sizeof(C) * (size_t)nblk * NB * NB);  // Linv blocks
  // err word, then two words (ticket, ready flag) per panel step
  // (then two more per 64-block for the first block of each middle panel)
  c->d_flags.ensure(std::max<size_t>(64, 4 * (4 + 4 * (size_t)nblk)));
  if (!c->stream2 || !c->stream3) {
    // the panel chain (context stream) first, then the lookahead updates,
    // then auxiliary work (right-hand sides, int8 operand planes), which only
    // fills SMs the factorisation leaves idle
    int least = 0, greatest = 0;
    DMB_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    const int mid = greatest < least ? greatest + 1 : least;
    if (!c->stream2) DMB_CUDA(cudaStreamCreateWithPriority(&c->stream2, cudaStreamNonBlocking, mid));
    if (!c->stream3) DMB_CUDA(cudaStreamCreateWithPriority(&c->stream3, cudaStreamNonBlocking, mid));
  }
  for (auto &e : c->la_ev)
    if (!e) DMB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  unsigned *err = c->d_flags.as<unsigned>();
  C *Linv = c->d_dinv.as<C>();
  unsigned *step_sync = err + 4;
  DMB_CUDA(cudaMemsetAsync(err, 0, 4 * (4 + 4 * (size_t)nblk), c->stream));
  // the fused panel step (strip + next diagonal block + next panel) for
  // complex64 factors; complex128 factors keep separate launches (their
  // 134 KB panel staging would allow one CTA per SM)
  const bool fuse_step = std::is_same<C, float2>::value;
  const size_t sm_panel = sizeof(C) * (2 * NB * (NB + 1) + NB);
  const size_t sm_step = std::max(sm_panel, diag_smem<C>());  // panel rows or the diagonal block
  const bool use_tc = std::is_same<C, float2>::value && dmb::tc_available(c);
  // trailing update F[r][cc] -= W[r][woff..woff+K) L[cc][jcol..jcol+K) on
  // rows >= r0, columns [r0, c_hi); slot: the packed-operand buffers of the
  // issuing stream (0 main, 1 stream2, 2 stream3)
  auto update = [&](int64_t r0, int64_t c_hi, int64_t jcol, int K, const C *Wb, int woff, int slot) {
    const int64_t rest = N - r0;
    if (rest <= 0 || c_hi <= r0) return;
    kt_begin(c);
    if (use_tc) {
      dmb::tc_ldlt_update_c64(c, N, r0, c_hi, jcol, K, (float2 *)F, (const float2 *)Wb, NBW, woff, slot);
    } else if constexpr (std::is_same<C, double2>::value) {
      // complex128 factor: the FP64-pipe GEMM (128 x 64 tiles, lower triangle)
      dmb::zgemm64_lower_update(c, rest, c_hi - r0, K, (const double2 *)Wb + r0 * NBW + woff, NBW,
                                (const double2 *)F + r0 * N + jcol, N, (double2 *)F + r0 * N + r0, N);
    } else {
      dim3 g(blocks_for(rest, 64), blocks_for(c_hi - r0, 64));
      DMB_LAUNCH(c, k_ldlt_update<C>, g, 256, 0, N, r0, c_hi, jcol, K, F, Wb, NBW, woff, 0, (C *)nullptr, err);
    }
    // algorithmic work: K complex MACs per updated lower-triangle entry
    const double cols = (double)(c_hi - r0), rows = (double)rest;
    kt_end(c, 8.0 * K * (cols * rows - cols * (cols - 1) / 2.0), 2);
  };
  // Lookahead.  Updates of one panel are split by columns: the next 256
  // columns on the main stream (the next panel needs them), the rest of the
  // current 1024-wide block column on stream2 and, for the trailing update at
  // the end of a block column, everything beyond the next block column on
  // stream3.  Concurrent updates always cover disjoint column ranges; before
  // an update of columns that a side stream may still be updating, the main
  // stream joins that stream (pend2 / pend3).  Each stream packs into its own
  // buffer slot, and W is double-buffered per block column, so a stream3
  // update may run through the whole next block column.
  bool pend2 = false, pend3 = false;
  auto join2 = [&] {
    if (pend2) DMB_CUDA(cudaStreamWaitEvent(c->stream, c->la_ev[1], 0));
    pend2 = false;
  };
  auto join3 = [&] {
    if (pend3) DMB_CUDA(cudaStreamWaitEvent(c->stream, c->la_ev[3], 0));
    pend3 = false;
  };
  // columns [lo, hi) updated on a side stream (1: stream2, 2: stream3) after
  // everything issued so far on the main stream
  auto side = [&](int which, int64_t lo, int64_t hi, int64_t jcol, int K, const C *Wb, int woff) {
    if (lo >= hi || lo >= N) return;
    cudaStream_t s = which == 1 ? c->stream2 : c->stream3;
    cudaEvent_t start = c->la_ev[which == 1 ? 0 : 2], done = c->la_ev[which == 1 ? 1 : 3];
    DMB_CUDA(cudaEventRecord(start, c->stream));
    DMB_CUDA(cudaStreamWaitEvent(s, start, 0));
    {
      StreamSwap sw(c, s);
      update(lo, hi, jcol, K, Wb, woff, which);
    }
    DMB_CUDA(cudaEventRecord(done, s));
    (which == 1 ? pend2 : pend3) = true;
  };
  // after a 256-wide middle panel: the rest of its block column, and the
  // first 256 columns of the next block column (the next block column's first
  // panel): on stream3 behind the trailing update that also covers them, or,
  // after the block column's last panel, on the main stream once stream3 has
  // joined.  The trailing update at the block column's end then leaves those
  // 256 columns out, so no K = 1,024 update sits on the chain.
  auto update_block_column = [&](int64_t r0, int64_t c_hi, int64_t jcol, int K, const C *Wb, int woff) {
    join2();
    const int64_t cmid = std::min<int64_t>(c_hi, r0 + NBO);
    update(r0, cmid, jcol, K, Wb, woff, 0);
    side(1, cmid, c_hi, jcol, K, Wb, woff);
    const int64_t n0 = c_hi, n1 = std::min<int64_t>(N, c_hi + NBO);
    if (n0 < n1) {
      if (r0 >= c_hi) {  // the block column's last panel
        join3();
        update(n0, n1, jcol, K, Wb, woff, 0);
      } else {
        side(2, n0, n1, jcol, K, Wb, woff);
      }
    }
  };
  // after a block column: the trailing matrix beyond the next block column's
  // first panel
  auto update_trailing = [&](int64_t r0, int64_t jcol, int K, const C *Wb) {
    join2();
    join3();
    const int64_t c1 = std::min<int64_t>(N, r0 + NBO), c2 = std::min<int64_t>(N, r0 + NBW);
    side(1, c1, c2, jcol, K, Wb, 0);
    side(2, c2, N, jcol, K, Wb, 0);
  };
  int64_t bc = 0;
  for (int64_t J2 = 0; J2 < N; J2 += NBW, bc++) {
    C *Wb = c->d_W.as<C>() + (bc & 1) * N * NBW;
    const int64_t J2E = std::min<int64_t>(N, J2 + NBW);
    for (int64_t J = J2; J < J2E; J += NBO) {
      const int64_t JE = std::min<int64_t>(J2E, J + NBO);
      // diag_done / panel_done: the previous step's kernel already factored
      // this diagonal block / ran this panel
      bool diag_done = false, panel_done = false;
      for (int64_t j = J; j < JE; j += NB) {
        const int b = (int)std::min<int64_t>(NB, N - j);
        C *Lblk = Linv + (j / NB) * NB * NB;
        const int64_t rest = N - j - b;
        if constexpr (std::is_same<C, float2>::value) {
          if (!diag_done) {  // the first block of the middle panel: factor + panel rows in one launch
            DMB_LAUNCH(c, k_ldlt_first, 1 + blocks_for(std::max<int64_t>(rest, 0), NB), 256, sm_step, N, j, b, F,
                       Lblk, Wb, NBW, (int)(j - J2), step_sync + 2 * nblk + 2 * (j / NB), err);
            diag_done = panel_done = true;
          }
        }
        if (!diag_done) DMB_LAUNCH(c, k_ldlt_diag<C>, 1, 256, diag_smem<C>(), N, j, b, F, Lblk, err);
        if (rest <= 0) break;
        if (!panel_done)
          DMB_LAUNCH(c, k_ldlt_panel<C>, blocks_for(rest, NB), 256, sm_panel, N, j, b, F, Lblk, Wb, NBW,
                     (int)(j - J2));
        diag_done = panel_done = false;
        if (j + b < JE) {  // strip update inside the middle panel, fused with the next diagonal block
          const int nb_next = (int)std::min<int64_t>(NB, N - (j + b));
          dim3 g(blocks_for(rest, 64), blocks_for(JE - (j + b), 64));
          if (fuse_step) {
            DMB_LAUNCH(c, k_ldlt_step<C>, g.x * g.y, 256, sm_step, N, j + b, JE, j, b, F, Wb, NBW,
                       (int)(j - J2), (int)(j + b - J2), nb_next, Lblk + NB * NB, step_sync + 2 * (j / NB), err);
            panel_done = true;
          } else {
            DMB_LAUNCH(c, k_ldlt_update<C>, g, 256, 0, N, j + b, JE, j, b, F, Wb, NBW, (int)(j - J2), nb_next,
                       Lblk + NB * NB, err);
          }
          diag_done = true;
        }
      }
      update_block_column(JE, J2E, J, (int)(JE - J), Wb, (int)(J - J2));
    }
    update_trailing(J2E, J2, (int)(J2E - J2), Wb);
  }
  join2();
  join3();
  unsigned h_err = 0;
  DMB_CUDA(cudaMemcpyAsync(&h_err, err, 4, cudaMemcpyDeviceToHost, c->stream));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  DMB_REQUIRE(!(h_err & 4u), DMB_ERR_TIMEOUT, "factorisation: a panel-step wait expired");
  DMB_REQUIRE(h_err == 0, DMB_ERR_BREAKDOWN, "near-field factorisation broke down: zero or non-finite pivot");
  if (use_tc)
    DMB_REQUIRE(dmb::tc_error_word(c) == 0, DMB_ERR_TIMEOUT, "tensor-core update: a pipeline wait expired");
}

void ldlt_solve_blocked_c64(dmb_ctx *c, const float2 *F, double2 *x, int64_t R);

template <class C> void ldlt_solve(dmb_ctx *c, const C *F, double2 *x, int64_t R) {
  if constexpr (std::is_same<C, float2>::value) {
    // complex64 factor, one right-hand side: blocked sweeps with the 1024-row
    // block inverses (the flag-ordered sweeps below run a few columns
    // concurrently and are faster from two on)
    if (R == 1) {
      ldlt_solve_blocked_c64(c, F, x, R);
      return;
    }
  }
  const int64_t N = c->n;
  const int nblk = (int)((N + NB - 1) / NB);
  const size_t flag_words = (size_t)R * nblk + R;
  c->d_flags.ensure(std::max<size_t>(64, 4 * (flag_words + 2)));
  unsigned *err = c->d_flags.as<unsigned>();
  unsigned *tickets = err + 1;
  unsigned *flags = tickets + R;
  const C *Linv = c->d_dinv.as<C>();
  dim3 g(nblk, (unsigned)R);
  DMB_CUDA(cudaMemsetAsync(err, 0, 4 * (flag_words + 1), c->stream));
  set_smem_attrs<C>();
  const size_t sm = 2 * sizeof(C) * NB * NB;
  DMB_LAUNCH(c, k_trsv_fwd<C>, g, 256, sm, N, F, Linv, x, flags, tickets, err, c->spin_limit);
  DMB_LAUNCH(c, k_scale_by_dinv<C>, blocks_for(N * R, 256), 256, 0, N, R, F, x);
  DMB_CUDA(cudaMemsetAsync(tickets, 0, 4 * flag_words, c->stream));
  DMB_LAUNCH(c, k_trsv_bwd<C>, g, 256, sm, N, F, Linv, x, flags, tickets, err, c->spin_limit);
}

// ---------------------------------------------------------------------------
// Batched triangular solves for many right-hand sides (X column-major N x R).
// The factor is walked in 256-row panels: the in-panel part (four 64-blocks
// with their stored Linv) runs in k_trsm_panel, where one CTA owns TP_COLS
// right-hand sides; the rest of the rows receive one GEMM-shaped update per
// panel (tensor cores for the complex64 factor, SIMT otherwise).  F is read
// once per sweep instead of once per right-hand side.
// ---------------------------------------------------------------------------
constexpr int TP = 256;      // panel rows
constexpr int TP_COLS = 8;   // right-hand sides per CTA

// T[i][j] <- G(i, j) for i, j < 64 (zero outside bi x bj); TR reads G(j, i)
template <class FC, bool TR>
__device__ __forceinline__ void stage_tile(FC (*T)[65], const FC *__restrict__ G, int64_t ld, int bi, int bj) {
  for (int e = threadIdx.x; e < 64 * 64; e += 256) {
    const int a = e >> 6, b = e & 63;  // consecutive threads: consecutive b
    if (TR) {
      // element (i = b, j = a) = G[a * ld + b]
      T[b][a] = (b < bi && a < bj) ? G[(int64_t)a * ld + b] : FC{};
    } else {
      T[a][b] = (a < bi && b < bj) ? G[(int64_t)a * ld + b] : FC{};
    }
  }
}

template <class FC, bool BWD>
__global__ void __launch_bounds__(256) k_trsm_panel(int64_t N, int64_t R, int64_t p0, int width,
                                                    const FC *__restrict__ F, const FC *__restrict__ Linv,
                                                    double2 *__restrict__ X) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  FC(*T)[65] = reinterpret_cast<FC(*)[65]>(smem_raw);
  double2(*xs)[TP_COLS + 1] = reinterpret_cast<double2(*)[TP_COLS + 1]>(smem_raw + sizeof(FC) * 64 * 65);
  const int64_t r0 = (int64_t)blockIdx.x * TP_COLS;
  for (int e = threadIdx.x; e < width * TP_COLS; e += 256) {
    const int q = e / width, i = e % width;
    xs[i][q] = (r0 + q < R) ? X[(r0 + q) * N + p0 + i] : make_double2(0, 0);
  }
  const int nb = (width + 63) / 64;
  const int i = threadIdx.x & 63, qh = threadIdx.x >> 6;  // rows i, columns qh and qh + 4
  for (int s = 0; s < nb; s++) {
    const int b = BWD ? nb - 1 - s : s;
    const int bs = min(64, width - 64 * b);
    const int64_t t = (p0 >> 6) + b;  // global 64-block index
    __syncthreads();
    // BWD: x_b = Linv_b^T y_b, FWD: y_b = Linv_b x_b
    stage_tile<FC, BWD>(T, Linv + t * 4096, 64, bs, bs);
    __syncthreads();
    double2 acc0 = make_double2(0, 0), acc1 = make_double2(0, 0);
    if (i < bs) {
      for (int j = 0; j < bs; j++) {
        const double2 l = to_d2(T[i][j]);
        cfma(acc0, l, xs[64 * b + j][qh]);
        cfma(acc1, l, xs[64 * b + j][qh + 4]);
      }
    }
    __syncthreads();
    if (i < bs) {
      xs[64 * b + i][qh] = acc0;
      xs[64 * b + i][qh + 4] = acc1;
    }
    // the other blocks of the panel that depend on block b
    for (int s2 = s + 1; s2 < nb; s2++) {
      const int b2 = BWD ? nb - 1 - s2 : s2;
      const int bs2 = min(64, width - 64 * b2);
      __syncthreads();
      if (BWD)  // x_{b2} -= L[b, b2]^T x_b : T[i][j] = L[p0 + 64 b + j][p0 + 64 b2 + i]
        stage_tile<FC, true>(T, F + (p0 + 64 * b) * N + p0 + 64 * b2, N, bs2, bs);
      else      // y_{b2} -= L[b2, b] y_b  : T[i][j] = L[p0 + 64 b2 + i][p0 + 64 b + j]
        stage_tile<FC, false>(T, F + (p0 + 64 * b2) * N + p0 + 64 * b, N, bs2, bs);
      __syncthreads();
      if (i < bs2) {
        double2 u0 = make_double2(0, 0), u1 = make_double2(0, 0);
        for (int j = 0; j < bs; j++) {
          const double2 l = to_d2(T[i][j]);
          cfma(u0, l, xs[64 * b + j][qh]);
          cfma(u1, l, xs[64 * b + j][qh + 4]);
        }
        xs[64 * b2 + i][qh] = csub(xs[64 * b2 + i][qh], u0);
        xs[64 * b2 + i][qh + 4] = csub(xs[64 * b2 + i][qh + 4], u1);
      }
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < width * TP_COLS; e += 256) {
    const int q = e / width, ii = e % width;
    if (r0 + q < R) X[(r0 + q) * N + p0 + ii] = xs[ii][q];
  }
}

// SIMT panel update  Y[m, r] -= sum_k A(m, k) B[k, r]  (FP64 accumulation),
// A(m, k) = A[m lda + k] or, TR, A[k lda + m]; B, Y column-major.  64 x 64
// output tiles, K in chunks of 16.
template <class FC, bool TR>
__global__ void __launch_bounds__(256) k_gemm_sub(int64_t M, int64_t R, int K, const FC *__restrict__ A, int64_t lda,
                                                  const double2 *__restrict__ B, int64_t ldb, double2 *__restrict__ Y,
                                                  int64_t ldy) {
  __shared__ double2 As[16][65];
  __shared__ double2 Bs[16][65];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int64_t m0 = (int64_t)blockIdx.x * 64, r0 = (int64_t)blockIdx.y * 64;
  double2 acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b] = make_double2(0, 0);
  for (int k0 = 0; k0 < K; k0 += 16) {
    for (int e = threadIdx.x; e < 16 * 64; e += 256) {
      int kk, mm;
      if (TR) { mm = e & 63; kk = e >> 6; } else { kk = e & 15; mm = e >> 4; }
      const int64_t m = m0 + mm;
      const int kx = k0 + kk;
      As[kk][mm] = (m < M && kx < K) ? to_d2(TR ? A[(int64_t)kx * lda + m] : A[m * lda + kx]) : make_double2(0, 0);
      const int kb = e & 15, rb = e >> 4;
      const int64_t r = r0 + rb;
      Bs[kb][rb] = (r < R && k0 + kb < K) ? B[r * ldb + k0 + kb] : make_double2(0, 0);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; kk++) {
      double2 a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; u++) a[u] = As[kk][ty + 16 * u];
#pragma unroll
      for (int v = 0; v < 4; v++) b[v] = Bs[kk][tx + 16 * v];
#pragma unroll
      for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) cfma(acc[u][v], a[u], b[v]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; u++)
#pragma unroll
    for (int v = 0; v < 4; v++) {
      const int64_t m = m0 + ty + 16 * u, r = r0 + tx + 16 * v;
      if (m < M && r < R) Y[r * ldy + m] = csub(Y[r * ldy + m], acc[u][v]);
    }
}

template <class C> void trsm_panel_attrs() {
  static bool done = false;
  if (done) return;
  const int sm = (int)(sizeof(C) * 64 * 65 + sizeof(double2) * TP * (TP_COLS + 1));
  DMB_CUDA(cudaFuncSetAttribute(k_trsm_panel<C, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  DMB_CUDA(cudaFuncSetAttribute(k_trsm_panel<C, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  done = true;
}

// X[r_lo : r_hi] -= L[r_lo : r_hi, k_lo : k_lo + w] X[k_lo : k_lo + w]   (forward)
// X[r_lo : r_hi] -= L[k_lo : k_lo + w, r_lo : r_hi]^T X[k_lo : k_lo + w] (backward)
template <class C> void trsm_update(dmb_ctx *c, const C *F, int64_t N, int64_t r_lo, int64_t r_hi, int64_t k_lo,
                                    int w, bool bwd, double2 *X, int64_t R) {
  const int64_t M = r_hi - r_lo;
  if (M <= 0) return;
  if (std::is_same<C, float2>::value && R >= c->tc_min_rhs && dmb::tc_available(c)) {
    dmb::tc_trsm_update(c, (const float2 *)F, N, r_lo, r_hi, k_lo, w, bwd, X, R);
    return;
  }
  if constexpr (std::is_same<C, double2>::value) {
    if (M >= 128 && R >= 16) {  // complex128 factor: the FP64-pipe GEMM
      if (bwd)
        dmb::zgemm64_sub(c, true, M, R, w, F + k_lo * N + r_lo, N, X + k_lo, N, X + r_lo, N);
      else
        dmb::zgemm64_sub(c, false, M, R, w, F + r_lo * N + k_lo, N, X + k_lo, N, X + r_lo, N);
      return;
    }
  }
  dim3 g(blocks_for(M, 64), blocks_for(R, 64));
  if (bwd)
    DMB_LAUNCH(c, (k_gemm_sub<C, true>), g, 256, 0, M, R, w, F + k_lo * N + r_lo, N, X + k_lo, N, X + r_lo, N);
  else
    DMB_LAUNCH(c, (k_gemm_sub<C, false>), g, 256, 0, M, R, w, F + r_lo * N + k_lo, N, X + k_lo, N, X + r_lo, N);
}

// Two levels: 1024-row outer panels whose rows below (forward) / above
// (backward) receive one K = 1024 update, and inside each outer panel
// 256-row panels solved by k_trsm_panel with K = 256 updates restricted to
// the outer panel.
constexpr int TP_OUTER = 1024;

// forward solve restricted to rows [o0, o1): L[o0:o1, o0:o1] y = x
template <class C> void forward_block(dmb_ctx *c, const C *F, int64_t o0, int64_t o1, double2 *X, int64_t R) {
  const int64_t N = c->n;
  const size_t sm = sizeof(C) * 64 * 65 + sizeof(double2) * TP * (TP_COLS + 1);
  for (int64_t p0 = o0; p0 < o1; p0 += TP) {
    const int w = (int)std::min<int64_t>(TP, o1 - p0);
    DMB_LAUNCH(c, (k_trsm_panel<C, false>), blocks_for(R, TP_COLS), 256, sm, N, R, p0, w, F, c->d_dinv.as<C>(), X);
    trsm_update<C>(c, F, N, p0 + w, o1, p0, w, false, X, R);
  }
}

// Inverses of the 1024-row diagonal blocks of the unit lower factor by
// recursive doubling from the 64 x 64 block inverses of the factorisation:
// for consecutive s-blocks A, B inside one outer block,
//   [A 0; C B]^-1 = [A^-1 0; -B^-1 C A^-1  B^-1],
// s = 64, 128, 256, 512, all pairs of a level in one launch per product.
// X (column-major, leading dimension N; outer block o occupies rows o0..o1 and
// block-local columns 0..o1-o0) receives the inverses.

// X <- the 64-block inverses on the diagonal of every outer block, 0 elsewhere
__global__ void k_inv_init(int64_t N, const float2 *__restrict__ Linv, double2 *__restrict__ X) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N * TP_OUTER) return;
  const int64_t col = i / N, r = i % N;  // consecutive threads: consecutive rows
  const int64_t o0 = r - r % TP_OUTER;
  double2 v = make_double2(0.0, 0.0);
  if (o0 + col < N && (o0 + col) / NB == r / NB) {
    const float2 l = Linv[(r / NB) * NB * NB + (r % NB) * NB + (o0 + col) % NB];
    v = make_double2(l.x, l.y);
  }
  X[col * N + r] = v;
}

template <class TC> __device__ __forceinline__ TC inv_conv(double2 v);
template <> __device__ __forceinline__ float2 inv_conv<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }
template <> __device__ __forceinline__ double2 inv_conv<double2>(double2 v) { return v; }

// one product of a doubling level; pair slot y of outer block y / ppo covers
// A = [i0, i0 + s), B = [i0 + s, i0 + s + sb), i0 = o0 + 2 s (y % ppo)
//   STEP 1: T = F[B, A] (strict lower part of L) x A^-1     (sb x s)
//   STEP 2: X[B, A] = -B^-1 x T                             (sb x s)
// 64 x 64 output tiles (grid.x), FP32 SIMT with 16-deep shared stages
// TC: the arithmetic of the products (float2 for the tensor-core sweeps'
// inverses, double2 for the one-RHS sweeps')
template <int STEP, class TC = float2>
__global__ void __launch_bounds__(256) k_inv_level(int64_t N, int s, const float2 *__restrict__ F,
                                                   double2 *__restrict__ X, TC *__restrict__ T) {
  __shared__ TC As[16][65];
  __shared__ TC Bs[16][65];
  const int ppo = TP_OUTER / (2 * s);
  const int64_t o0 = (int64_t)(blockIdx.y / ppo) * TP_OUTER;
  const int64_t o1 = min(N, o0 + TP_OUTER);
  const int64_t i0 = o0 + 2 * (int64_t)s * (blockIdx.y % ppo);
  const int64_t a0 = i0, b0 = i0 + s;
  if (b0 >= o1) return;  // no B block in this slot
  const int sb = (int)min((int64_t)s, o1 - b0);
  const int nt = (s + 63) / 64;
  const int ti = blockIdx.x / nt, tj = blockIdx.x % nt;
  if (64 * ti >= sb) return;
  TC *Tp = T + (int64_t)blockIdx.y * s * s;  // column-major sb x s, leading dimension s
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  TC acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = czero<TC>();
  // STEP 1: k runs over A's columns from the tile's first column (A^-1 is
  // lower); STEP 2: over B's columns up to the tile's last row (B^-1 is lower)
  const int k_lo = STEP == 1 ? 64 * tj : 0;
  const int k_hi = STEP == 1 ? s : min(sb, 64 * ti + 64);
  for (int k0 = k_lo; k0 < k_hi; k0 += 16) {
    for (int e = threadIdx.x; e < 16 * 64; e += 256) {
      if (STEP == 1) {
        const int kk = e & 15, rr = e >> 4;  // k fastest: F rows and X columns are k-contiguous
        const int k = k0 + kk, i = 64 * ti + rr, j = 64 * tj + rr;
        const float2 f = (k < k_hi && i < sb) ? F[(b0 + i) * N + a0 + k] : make_float2(0.f, 0.f);
        As[kk][rr] = inv_conv<TC>(make_double2(f.x, f.y));
        const double2 x = (k < k_hi) ? X[(a0 - o0 + j) * N + a0 + k] : make_double2(0.0, 0.0);
        Bs[kk][rr] = inv_conv<TC>(x);
      } else {
        const int rr = e & 63, kk = e >> 6;  // rows fastest for B^-1 (column-major)
        const int k = k0 + kk, i = 64 * ti + rr;
        const double2 x = (k < k_hi && i < sb) ? X[(b0 - o0 + k) * N + b0 + i] : make_double2(0.0, 0.0);
        As[kk][rr] = inv_conv<TC>(x);
        const int kk2 = e & 15, cc = e >> 4, k2 = k0 + kk2, j = 64 * tj + cc;
        Bs[kk2][cc] = (k2 < k_hi && j < s) ? Tp[(int64_t)j * s + k2] : czero<TC>();
      }
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; kk++) {
      TC a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) cfma(acc[i][j], a[i], b[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int r = 64 * ti + ty + 16 * i, cidx = 64 * tj + tx + 16 * j;
      if (r >= sb || cidx >= s) continue;
      if (STEP == 1)
        Tp[(int64_t)cidx * s + r] = acc[i][j];
      else
        X[(a0 - o0 + cidx) * N + b0 + r] = make_double2(-(double)acc[i][j].x, -(double)acc[i][j].y);
    }
}

// Pack the complex64 factor for the tensor-core sweeps (once per
// factorisation): L'' and (L^T)'', and the inverses of the 1024-row diagonal
// blocks of L (recursive doubling, k_inv_init / k_inv_level).
// The 1024-row block inverses of L (once per factorisation): FP32 products
// into d_trsm_id for the tensor-core sweeps (which round them to TF32
// anyway), FP64 products into d_sv_inv for the one-RHS sweeps (as accurate as
// substitution with the stored 64-block inverses).
template <class TC> void prepare_block_inverses(dmb_ctx *c, const float2 *F) {
  constexpr bool f64 = std::is_same<TC, double2>::value;
  uint64_t &ver = f64 ? c->f_inv64 : c->f_inv;
  if (ver == c->f_version) return;
  const int64_t N = c->n;
  DevBuf &dst = f64 ? c->d_sv_inv : c->d_trsm_id;
  dst.ensure(sizeof(double2) * N * TP_OUTER);
  double2 *Xid = dst.as<double2>();
  const int64_t nout = (N + TP_OUTER - 1) / TP_OUTER;
  // scratch for the products T: (pair slots) x s x s <= nout x 1024 x 256
  c->d_trsm_t.ensure(sizeof(TC) * nout * TP_OUTER * (TP_OUTER / 4));
  TC *T = c->d_trsm_t.as<TC>();
  DMB_LAUNCH(c, k_inv_init, blocks_for(N * TP_OUTER, 256), 256, 0, N, c->d_dinv.as<float2>(), Xid);
  for (int s = NB; s < TP_OUTER; s *= 2) {
    const int nt = (s + 63) / 64;
    dim3 g((unsigned)(nt * nt), (unsigned)(nout * (TP_OUTER / (2 * s))));
    DMB_LAUNCH(c, (k_inv_level<1, TC>), g, 256, 0, N, s, F, Xid, T);
    DMB_LAUNCH(c, (k_inv_level<2, TC>), g, 256, 0, N, s, F, Xid, T);
  }
  ver = c->f_version;
}

void prepare_packed_factor(dmb_ctx *c, const float2 *F) {
  if (c->f_packed == c->f_version) return;
  const int64_t N = c->n;
  trsm_panel_attrs<float2>();
  dmb::tc_trsm_pack_factor(c, F, N);
  prepare_block_inverses<float2>(c, F);
  double2 *Xid = c->d_trsm_id.as<double2>();
  const int64_t nout = (N + TP_OUTER - 1) / TP_OUTER;
  for (int64_t o = 0; o < nout; o++) {
    const int64_t o0 = o * TP_OUTER, o1 = std::min<int64_t>(N, o0 + TP_OUTER);
    dmb::tc_trsm_pack_diag(c, o, Xid + o0, N, (int)(o1 - o0));
  }
  c->f_packed = c->f_version;
}

// ---------------------------------------------------------------------------
// One-RHS sweeps of a complex64 factor with the 1024-row block inverses X_o:
//   forward, o = 0, 1, ...:  a = b_o - L[o, <o] y;   y_o = X_o a
//   backward, o = last..0:   a = z_o - L[>o, o]^T x; x_o = X_o^T a
// Eleven block steps per sweep at N = 10,680, each two or three launches of
// bandwidth-bound products (L read once per sweep, X_o once); no waits
// between CTAs, fixed summation order.
// ---------------------------------------------------------------------------
constexpr int SV_IC = 64;  // rows per partial-sum chunk of the column products

// y[i] = (SUB ? b[i] - s : s), s = sum_j M[i ld + j] v[j], i < rows: a warp per row
template <class MC, bool SUB>
__global__ void __launch_bounds__(256) k_sv_rowdot(int rows, int cols, const MC *__restrict__ M, int64_t ld,
                                                   const double2 *__restrict__ v, const double2 *__restrict__ b,
                                                   double2 *__restrict__ y) {
  const int i = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (i >= rows) return;
  const MC *Mi = M + (int64_t)i * ld;
  // four loads in flight per lane (one warp per row leaves few warps)
  double2 a0 = make_double2(0, 0), a1 = make_double2(0, 0), a2 = make_double2(0, 0), a3 = make_double2(0, 0);
  int j = lane;
  for (; j + 96 < cols; j += 128) {
    cfma(a0, to_d2(Mi[j]), v[j]);
    cfma(a1, to_d2(Mi[j + 32]), v[j + 32]);
    cfma(a2, to_d2(Mi[j + 64]), v[j + 64]);
    cfma(a3, to_d2(Mi[j + 96]), v[j + 96]);
  }
  for (; j < cols; j += 32) cfma(a0, to_d2(Mi[j]), v[j]);
  a0 = warp_sum2(cadd(cadd(a0, a1), cadd(a2, a3)));
  if (lane == 0) y[i] = SUB ? csub(b[i], a0) : a0;
}

// part[chunk][j] = sum over the chunk's rows i of M[i ld + j] v[i], j < ncols
// (chunk = blockIdx.y, SV_IC rows; consecutive threads read consecutive j)
template <class MC>
__global__ void __launch_bounds__(256) k_sv_colpart(int nrows, int ncols, const MC *__restrict__ M, int64_t ld,
                                                    const double2 *__restrict__ v, double2 *__restrict__ part) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ncols) return;
  const int i0 = blockIdx.y * SV_IC, i1 = min(nrows, i0 + SV_IC);
  double2 a0 = make_double2(0, 0), a1 = make_double2(0, 0);
  int i = i0;
  for (; i + 1 < i1; i += 2) {
    cfma(a0, to_d2(M[(int64_t)i * ld + j]), v[i]);
    cfma(a1, to_d2(M[(int64_t)(i + 1) * ld + j]), v[i + 1]);
  }
  if (i < i1) cfma(a0, to_d2(M[(int64_t)i * ld + j]), v[i]);
  part[(int64_t)blockIdx.y * ncols + j] = cadd(a0, a1);
}

// y[j] = (sub ? b[j] - s : s), s = the chunks' partial sums in order
__global__ void k_sv_colsum(int ncols, int nchunks, const double2 *__restrict__ part, const double2 *__restrict__ b,
                            int sub, double2 *__restrict__ y) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ncols) return;
  double2 s = make_double2(0, 0);
  for (int q = 0; q < nchunks; q++) s = cadd(s, part[(int64_t)q * ncols + j]);
  y[j] = sub ? csub(b[j], s) : s;
}

void ldlt_solve_blocked_c64(dmb_ctx *c, const float2 *F, double2 *x, int64_t R) {
  const int64_t N = c->n;
  prepare_block_inverses<double2>(c, F);
  const double2 *X = c->d_sv_inv.as<double2>();
  const int64_t nout = (N + TP_OUTER - 1) / TP_OUTER;
  const int max_chunks = (int)std::max<int64_t>((N + SV_IC - 1) / SV_IC, 1);
  c->d_sv_acc.ensure(sizeof(double2) * TP_OUTER);
  c->d_sv_part.ensure(sizeof(double2) * (size_t)max_chunks * TP_OUTER);
  double2 *acc = c->d_sv_acc.as<double2>(), *part = c->d_sv_part.as<double2>();
  for (int64_t r = 0; r < R; r++) {
    double2 *xr = x + r * N;
    for (int64_t o = 0; o < nout; o++) {  // forward
      const int64_t o0 = o * TP_OUTER;
      const int w = (int)std::min<int64_t>(TP_OUTER, N - o0);
      const double2 *a = xr + o0;
      if (o0 > 0) {
        DMB_LAUNCH(c, (k_sv_rowdot<float2, true>), blocks_for((int64_t)w * 32, 256), 256, 0, w, (int)o0,
                   F + o0 * N, N, xr, xr + o0, acc);
        a = acc;
      }
      const int nch = (w + SV_IC - 1) / SV_IC;
      // y_o[i] = sum_k X_o[i][k] a[k]; X_o column k is contiguous: X[k N + o0 + i]
      DMB_LAUNCH(c, k_sv_colpart<double2>, dim3(blocks_for(w, 256), (unsigned)nch), 256, 0, w, w, X + o0, N, a,
                 part);
      DMB_LAUNCH(c, k_sv_colsum, blocks_for(w, 256), 256, 0, w, nch, part, (const double2 *)nullptr, 0, xr + o0);
    }
    DMB_LAUNCH(c, k_scale_by_dinv<float2>, blocks_for(N, 256), 256, 0, N, (int64_t)1, F, xr);
    for (int64_t o = nout - 1; o >= 0; o--) {  // backward
      const int64_t o0 = o * TP_OUTER, o1 = std::min<int64_t>(N, o0 + TP_OUTER);
      const int w = (int)(o1 - o0);
      const double2 *a = xr + o0;
      if (o1 < N) {
        // a[c] = z[o0 + c] - sum_{i >= o1} L[i][o0 + c] x[i]
        const int nr = (int)(N - o1), nch = (nr + SV_IC - 1) / SV_IC;
        DMB_LAUNCH(c, k_sv_colpart<float2>, dim3(blocks_for(w, 256), (unsigned)nch), 256, 0, nr, w,
                   F + o1 * N + o0, N, xr + o1, part);
        DMB_LAUNCH(c, k_sv_colsum, blocks_for(w, 256), 256, 0, w, nch, part, xr + o0, 1, acc);
        a = acc;
      }
      // x_o[k] = sum_i X_o[i][k] a[i] = sum_i X[k N + o0 + i] a[i]: a warp per output
      if (a == acc) {
        DMB_LAUNCH(c, (k_sv_rowdot<double2, false>), blocks_for((int64_t)w * 32, 256), 256, 0, w, w, X + o0, N, a,
                   (const double2 *)nullptr, xr + o0);
      } else {
        // the last block reads and writes x_o: go through the scratch vector
        DMB_CUDA(cudaMemcpyAsync(acc, xr + o0, sizeof(double2) * w, cudaMemcpyDeviceToDevice, c->stream));
        DMB_LAUNCH(c, (k_sv_rowdot<double2, false>), blocks_for((int64_t)w * 32, 256), 256, 0, w, w, X + o0, N,
                   acc, (const double2 *)nullptr, xr + o0);
      }
    }
  }
}

template <class C> void ldlt_solve_batched(dmb_ctx *c, const C *F, double2 *X, int64_t R) {
  const int64_t N = c->n;
  const C *Linv = c->d_dinv.as<C>();
  trsm_panel_attrs<C>();
  if (std::is_same<C, float2>::value && R >= c->tc_min_rhs && dmb::tc_available(c)) {
    // tensor cores: every step is a GEMM on operands packed once per factor
    prepare_packed_factor(c, (const float2 *)F);
    dmb::tc_trsm_sweep(c, N, X, R, false);
    DMB_LAUNCH(c, k_scale_by_dinv<C>, blocks_for(N * R, 256), 256, 0, N, R, F, X);
    dmb::tc_trsm_sweep(c, N, X, R, true);
    return;
  }
  const size_t sm = sizeof(C) * 64 * 65 + sizeof(double2) * TP * (TP_COLS + 1);
  const unsigned gcols = blocks_for(R, TP_COLS);
  const int64_t nout = (N + TP_OUTER - 1) / TP_OUTER;
  for (int64_t o = 0; o < nout; o++) {
    const int64_t o0 = o * TP_OUTER, o1 = std::min<int64_t>(N, o0 + TP_OUTER);
    forward_block<C>(c, F, o0, o1, X, R);
    trsm_update<C>(c, F, N, o1, N, o0, (int)(o1 - o0), false, X, R);
  }
  DMB_LAUNCH(c, k_scale_by_dinv<C>, blocks_for(N * R, 256), 256, 0, N, R, F, X);
  for (int64_t o = nout - 1; o >= 0; o--) {
    const int64_t o0 = o * TP_OUTER, o1 = std::min<int64_t>(N, o0 + TP_OUTER);
    const int64_t np = (o1 - o0 + TP - 1) / TP;
    for (int64_t pi = np - 1; pi >= 0; pi--) {
      const int64_t p0 = o0 + pi * TP;
      const int w = (int)std::min<int64_t>(TP, o1 - p0);
      DMB_LAUNCH(c, (k_trsm_panel<C, true>), gcols, 256, sm, N, R, p0, w, F, Linv, X);
      trsm_update<C>(c, F, N, o0, p0, p0, w, true, X, R);
    }
    trsm_update<C>(c, F, N, 0, o0, o0, (int)(o1 - o0), true, X, R);
  }
}

}  // namespace

namespace dmb {

unsigned read_err_word(dmb_ctx *c) {
  unsigned e = 0;
  if (!c->d_flags.p) return 0;  // no triangular solve has run on this context
  DMB_CUDA(cudaMemcpyAsync(&e, c->d_flags.p, 4, cudaMemcpyDeviceToHost, c->stream));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  return e;
}

void nf_build(dmb_ctx *c, double cutoff, int kind) {
  double t0 = now_ms();
  const int64_t N = c->n;
  const bool f64 = c->z_prec == DMB_PREC_FP64;
  c->pc_valid = false;
  if (kind == DMB_PRECOND_NF_DIAG) {
    DevBuf tmp;
    tmp.ensure(16);
    DMB_CUDA(cudaMemsetAsync(tmp.p, 0, 16, c->stream));
    c->d_dinv.ensure(sizeof(double2) * N);
    unsigned *bad = (unsigned *)(tmp.as<double>() + 1);
    if (f64) {
      DMB_LAUNCH(c, k_diag_max<double2>, 1, 1024, 0, N, c->d_Z.as<double2>(), tmp.as<double>(), bad);
      DMB_LAUNCH(c, k_diag_inv<double2>, blocks_for(N, 256), 256, 0, N, c->d_Z.as<double2>(), tmp.as<double>(),
                 c->d_dinv.as<double2>());
    } else {
      DMB_LAUNCH(c, k_diag_max<float2>, 1, 1024, 0, N, c->d_Z.as<float2>(), tmp.as<double>(), bad);
      DMB_LAUNCH(c, k_diag_inv<float2>, blocks_for(N, 256), 256, 0, N, c->d_Z.as<float2>(), tmp.as<double>(),
                 c->d_dinv.as<double2>());
    }
    double mx[2];
    DMB_CUDA(cudaMemcpyAsync(mx, tmp.p, 16, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
    unsigned hb;
    memcpy(&hb, &mx[1], 4);
    DMB_REQUIRE(hb == 0, DMB_ERR_ARGUMENT, "near-field diagonal entries must be finite");
    DMB_REQUIRE(mx[0] > 0, DMB_ERR_ARGUMENT, "cannot build a diagonal preconditioner from an all-zero diagonal");
    c->nnz_ratio = 1.0 / (double)N;
    c->pc_kind = kind;
    c->pc_prec = c->z_prec;
    c->pc_valid = true;
    c->tm.precond_ms = now_ms() - t0;
    return;
  }
  size_t esz = f64 ? sizeof(double2) : sizeof(float2);
  c->d_F.ensure(esz * N * N);
  c->d_small.ensure(65536);
  DevBuf cnt;  // view into the persistent scratch (first 8 bytes), not owned
  cnt.p = c->d_small.p;
  DMB_CUDA(cudaMemsetAsync(cnt.p, 0, 8, c->stream));
  if (!std::isfinite(cutoff) && cutoff > 0) {
    // every entry is kept: a plain device copy of Z
    DMB_CUDA(cudaMemcpyAsync(c->d_F.p, c->d_Z.p, esz * N * N, cudaMemcpyDeviceToDevice, c->stream));
    c->nnz_ratio = 1.0;
  } else {
    dim3 g(blocks_for(N, 32), blocks_for(N, 32));
    if (f64)
      DMB_LAUNCH(c, (k_nf_mask<double2, double2>), g, 256, 0, N, c->d_Z.as<double2>(), c->d_centers.as<double>(),
                 cutoff, c->d_F.as<double2>(), cnt.as<unsigned long long>());
    else
      DMB_LAUNCH(c, (k_nf_mask<float2, float2>), g, 256, 0, N, c->d_Z.as<float2>(), c->d_centers.as<double>(),
                 cutoff, c->d_F.as<float2>(), cnt.as<unsigned long long>());
    unsigned long long h_cnt = 0;
    DMB_CUDA(cudaMemcpyAsync(&h_cnt, cnt.p, 8, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
    c->nnz_ratio = ((double)h_cnt / (double)N) / (double)N;
  }
  if (f64)
    ldlt_factor(c, c->d_F.as<double2>());
  else
    ldlt_factor(c, c->d_F.as<float2>());
  c->pc_kind = kind;
  c->pc_prec = c->z_prec;
  c->pc_valid = true;
  c->tm.precond_ms = now_ms() - t0;
}

// factor a near-field matrix already written to d_F (precision of its
// storage) and make it the context's preconditioner
void nf_factor_resident(dmb_ctx *c, int kind, int precision) {
  c->pc_valid = false;
  if (precision == DMB_PREC_FP64)
    ldlt_factor(c, c->d_F.as<double2>());
  else
    ldlt_factor(c, c->d_F.as<float2>());
  c->pc_kind = kind;
  c->pc_prec = precision;
  c->pc_valid = true;
}

void pc_apply_dev(dmb_ctx *c, double *x, int64_t nrhs) {
  DMB_REQUIRE(c->pc_valid, DMB_ERR_STATE, "no preconditioner built");
  const int64_t N = c->n;
  double2 *xd = (double2 *)x;
  if (c->pc_kind == DMB_PRECOND_NF_DIAG) {
    DMB_LAUNCH(c, k_scale_vec, blocks_for(N * nrhs, 256), 256, 0, N, nrhs, c->d_dinv.as<double2>(), xd);
    return;
  }
  if (c->pc_kind == DMB_PRECOND_NF_LU) {
    // one right-hand side at a time streams F per column; from 8 columns on
    // the panel-blocked solves read F once per sweep
    const bool batched = nrhs >= 8;
    if (c->pc_prec == DMB_PREC_FP64) {
      if (batched) ldlt_solve_batched(c, c->d_F.as<double2>(), xd, nrhs);
      else ldlt_solve(c, c->d_F.as<double2>(), xd, nrhs);
    } else {
      if (batched) ldlt_solve_batched(c, c->d_F.as<float2>(), xd, nrhs);
      else ldlt_solve(c, c->d_F.as<float2>(), xd, nrhs);
    }
    return;
  }
  if (c->pc_kind == DMB_PRECOND_LOCAL_INV || c->pc_kind == DMB_PRECOND_LEARNED || c->pc_kind == DMB_PRECOND_RING) {
    dmb::local_apply_dev(c, x, nrhs);
    return;
  }
  throw DmbError{DMB_ERR_STATE, "preconditioner kind not available"};
}

}  // namespace dmb
