// dmb_linalg.cu -- dense operators on the resident impedance matrix:
//   * Z*x (the zgemv Krylov.gmres performs every iteration) and Z*X,
//   * near-field matrix extraction (NearFieldPreconditioner.jl:247-369,
//     429-464, 670-716) and its factorisation,
//   * triangular solves of the preconditioner apply (NearFieldOperator,
//     NearFieldPreconditioner.jl:1034-1054),
//   * direct solve with FP64 iterative refinement (Solve.jl:1124-1198).
//
// Factorisation.  The near-field matrix of a complex-symmetric EFIE system is
// itself complex symmetric, so it is factored as Z_nf = L D L^T (unit lower L,
// diagonal D, no pivoting) -- the same inverse as UMFPACK's sparse LU up to
// rounding, at half the flops of LU.  A zero or non-finite pivot stops the
// factorisation with DMB_ERR_BREAKDOWN instead of returning garbage.
//
// Triangular solves run as ONE kernel per sweep: each CTA draws a ticket
// (block row, in launch order), subtracts the contributions of the block rows
// already solved as soon as their flags are published, then applies the
// precomputed inverse of its unit-lower diagonal block.  Every wait is bounded:
// on expiry the kernel records DMB_ERR_TIMEOUT in an error word and returns.
#include <algorithm>
#include <cmath>

#include "dmb_device.cuh"
#include "dmb_internal.h"

namespace {

constexpr int NB = 32;   // factorisation panel width
constexpr int SB = 64;   // triangular-solve block
constexpr long long SPIN_LIMIT = 20000000;  // ~2-4 s with nanosleep

// ---------------------------------------------------------------------------
// matvec
// ---------------------------------------------------------------------------
// y = Z x for one right-hand side: one warp per row, 16-byte loads.
template <class ZC>
__global__ void k_gemv(int64_t N, const ZC *__restrict__ Z, const double2 *__restrict__ x,
                       double2 *__restrict__ y) {
  int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  int lane = threadIdx.x & 31;
  if (row >= N) return;
  const ZC *zr = Z + row * N;
  double re = 0, im = 0;
  for (int64_t n = lane; n < N; n += 32) {
    double2 z = to_d2(zr[n]);
    double2 v = x[n];
    re = fma(z.x, v.x, re);
    re = fma(-z.y, v.y, re);
    im = fma(z.x, v.y, im);
    im = fma(z.y, v.x, im);
  }
  re = warp_sum(re);
  im = warp_sum(im);
  if (lane == 0) y[row] = make_double2(re, im);
}

// Y = Z X for R right-hand sides (X, Y column-major N x R), SIMT tiles with
// FP64 accumulation.  64 x 64 output tile, 16-deep K chunks.
template <class ZC>
__global__ void __launch_bounds__(256) k_gemm_zx(int64_t N, int64_t R, const ZC *__restrict__ Z,
                                                 const double2 *__restrict__ X,
                                                 double2 *__restrict__ Y) {
  __shared__ double2 As[16][65];
  __shared__ double2 Bs[16][65];
  int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  int64_t m0 = (int64_t)blockIdx.x * 64, r0 = (int64_t)blockIdx.y * 64;
  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = make_double2(0, 0);
  for (int64_t k0 = 0; k0 < N; k0 += 16) {
    for (int e = threadIdx.x; e < 16 * 64; e += 256) {
      int kk = e & 15, mm = e >> 4;
      int64_t m = m0 + mm, kx = k0 + kk;
      As[kk][mm] = (m < N && kx < N) ? to_d2(Z[m * N + kx]) : make_double2(0, 0);
      int64_t r = r0 + mm;
      Bs[kk][mm] = (r < R && kx < N) ? X[r * N + kx] : make_double2(0, 0);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; kk++) {
      double2 a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
          acc[i][j].x = fma(a[i].x, b[j].x, acc[i][j].x);
          acc[i][j].x = fma(-a[i].y, b[j].y, acc[i][j].x);
          acc[i][j].y = fma(a[i].x, b[j].y, acc[i][j].y);
          acc[i][j].y = fma(a[i].y, b[j].x, acc[i][j].y);
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      int64_t m = m0 + ty + 16 * i, r = r0 + tx + 16 * j;
      if (m < N && r < R) Y[r * N + m] = acc[i][j];
    }
}

// ---------------------------------------------------------------------------
// Z out / entries / conversions
// ---------------------------------------------------------------------------
__global__ void k_f2_to_d2(int64_t count, const float2 *__restrict__ a, double2 *__restrict__ b) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) b[i] = make_double2(a[i].x, a[i].y);
}

template <class ZC>
__global__ void k_entries(int64_t count, int64_t N, const int64_t *__restrict__ mn, const ZC *__restrict__ Z,
                          double2 *__restrict__ out) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  out[i] = to_d2(Z[(mn[2 * i] - 1) * N + (mn[2 * i + 1] - 1)]);
}

// ---------------------------------------------------------------------------
// impedance loading: Z[m][n] -= zs_t * sum_q w_q f_m.f_n 2A_t
// ---------------------------------------------------------------------------
template <class ZC>
__global__ void k_impedance_offdiag(int nt, const TriCache *__restrict__ tc, int nq,
                                    const double *__restrict__ wq, const double2 *__restrict__ zs,
                                    int64_t N, ZC *__restrict__ Z) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const TriCache &T = tc[t];
  double2 th = zs[t];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      int m = T.rwg[i], n = T.rwg[j];
      if (m < 0 || n < 0 || m == n) continue;
      double v = 0;
      for (int q = 0; q < nq; q++) {
        double fa[3], fb[3];
        for (int d = 0; d < 3; d++) {
          fa[d] = T.s[i] * (T.qp[q][d] - T.p[i][d]);
          fb[d] = T.s[j] * (T.qp[q][d] - T.p[j][d]);
        }
        v += wq[q] * (fa[0] * fb[0] + fa[1] * fb[1] + fa[2] * fb[2]);
      }
      v *= 2 * T.area;
      ZC *p = Z + (int64_t)m * N + n;
      store_c(p, csub(to_d2(*p), cscale(th, v)));
    }
}

template <class ZC>
__global__ void k_impedance_diag(int64_t N, const TriCache *__restrict__ tc, const int *__restrict__ rslot,
                                 int nq, const double *__restrict__ wq, const double2 *__restrict__ zs,
                                 ZC *__restrict__ Z) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= N) return;
  double2 acc = to_d2(Z[m * N + m]);
  for (int s = 0; s < 2; s++) {
    int sl = rslot[2 * m + s];
    int t = sl / 3, i = sl % 3;
    const TriCache &T = tc[t];
    double v = 0;
    for (int q = 0; q < nq; q++) {
      double f[3];
      for (int d = 0; d < 3; d++) f[d] = T.s[i] * (T.qp[q][d] - T.p[i][d]);
      v += wq[q] * (f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    }
    v *= 2 * T.area;
    acc = csub(acc, cscale(zs[t], v));
  }
  store_c(Z + m * N + m, acc);
}

// ---------------------------------------------------------------------------
// near-field extraction (cutoff on RWG centre distance, inclusive)
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool within_cutoff(const double *a, const double *b, double cutoff) {
  if (!isfinite(cutoff)) return true;
  double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  double d = hypot(hypot(dx, dy), dz);
  if (d != cutoff) return d <= cutoff;
  // exact tie-break (NearFieldPreconditioner.jl:339-355): compare the exact
  // squared distance with cutoff^2 in double-double
  double s = 0, e = 0;
  double v[3] = {dx, dy, dz};
  for (int i = 0; i < 3; i++) {
    double p = v[i] * v[i], pe = fma(v[i], v[i], -p);
    double t = s + p, bb = t - s;
    e += (s - (t - bb)) + (p - bb) + pe;
    s = t;
  }
  double c2 = cutoff * cutoff, c2e = fma(cutoff, cutoff, -c2);
  return (s - c2) + (e - c2e) <= 0.0;
}

template <class ZC, class FC>
__global__ void k_nf_mask(int64_t N, const ZC *__restrict__ Z, const double *__restrict__ cen,
                          double cutoff, FC *__restrict__ F, unsigned long long *__restrict__ nnz) {
  int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t m = blockIdx.y;
  unsigned keep = 0;
  if (n < N) {
    bool k;
    if (cutoff <= 0.0) k = (m == n);
    else k = (m == n) || within_cutoff(cen + 3 * m, cen + 3 * n, cutoff);
    double2 z = k ? to_d2(Z[m * N + n]) : make_double2(0, 0);
    store_c(F + m * N + n, z);
    keep = k;
  }
  unsigned cnt = __reduce_add_sync(0xffffffffu, keep);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(nnz, (unsigned long long)cnt);
}

template <class ZC>
__global__ void k_diag_max(int64_t N, const ZC *__restrict__ Z, double *__restrict__ out,
                           unsigned *__restrict__ bad) {
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

// Jacobi with the 1e-10 * max|z_ii| floor (NearFieldPreconditioner.jl:623-668)
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
// LDL^T (complex symmetric, unpivoted), lower triangle of row-major F
// ---------------------------------------------------------------------------
template <class FC>
__global__ void k_ldlt_diag(int64_t N, int64_t j, int b, FC *__restrict__ F, unsigned *__restrict__ err) {
  __shared__ double2 A[NB][NB + 1];
  for (int e = threadIdx.x; e < b * b; e += blockDim.x) {
    int i = e / b, c = e % b;
    A[i][c] = (c <= i) ? to_d2(F[(j + i) * N + j + c]) : make_double2(0, 0);
  }
  __syncthreads();
  for (int k = 0; k < b; k++) {
    double2 d = A[k][k];
    double ad = hypot(d.x, d.y);
    if (!(ad > 0.0) || !isfinite(ad)) {
      if (threadIdx.x == 0) atomicOr(err, 2u);
      return;
    }
    // trailing update of the diagonal block: A[i][c] -= A[i][k] * A[c][k] / d
    for (int e = threadIdx.x; e < b * b; e += blockDim.x) {
      int i = e / b, c = e % b;
      if (c > k && c <= i) {
        double2 lc = cdiv(A[c][k], d);
        A[i][c] = csub(A[i][c], cmul(A[i][k], lc));
      }
    }
    __syncthreads();
    for (int i = k + 1 + threadIdx.x; i < b; i += blockDim.x) A[i][k] = cdiv(A[i][k], d);
    __syncthreads();
  }
  for (int e = threadIdx.x; e < b * b; e += blockDim.x) {
    int i = e / b, c = e % b;
    if (c <= i) store_c(F + (j + i) * N + j + c, A[i][c]);
  }
}

// rows r >= j+b: y L11^T = a (forward substitution across the warp), then
// W[r] = y (= L21 D1 row), L21[r] = y / D1.
template <class FC>
__global__ void k_ldlt_panel(int64_t N, int64_t j, int b, FC *__restrict__ F, double2 *__restrict__ W) {
  __shared__ double2 L[NB][NB + 1];
  for (int e = threadIdx.x; e < b * b; e += blockDim.x) {
    int i = e / b, c = e % b;
    L[i][c] = (c <= i) ? to_d2(F[(j + i) * N + j + c]) : make_double2(0, 0);
  }
  __syncthreads();
  int lane = threadIdx.x & 31;
  int64_t r = j + b + (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (r >= N) return;
  double2 a = lane < b ? to_d2(F[r * N + j + lane]) : make_double2(0, 0);
  for (int c = 0; c < b; c++) {
    double yr = __shfl_sync(0xffffffffu, a.x, c), yi = __shfl_sync(0xffffffffu, a.y, c);
    if (lane > c && lane < b) a = csub(a, cmul(make_double2(yr, yi), L[lane][c]));
  }
  if (lane < b) {
    W[r * NB + lane] = a;
    store_c(F + r * N + j + lane, cdiv(a, L[lane][lane]));
  }
}

__device__ __forceinline__ void lower_tile(int64_t t, int T, int &bi, int &bj) {
  // enumerate tiles (bi >= bj) row by row: row bi has bi+1 tiles
  int i = (int)floor((sqrt(8.0 * (double)t + 1.0) - 1.0) / 2.0);
  while ((int64_t)i * (i + 1) / 2 > t) i--;
  while ((int64_t)(i + 1) * (i + 2) / 2 <= t) i++;
  bi = i;
  bj = (int)(t - (int64_t)i * (i + 1) / 2);
}

// C[r][c] -= sum_k W[r][k] L[c][k]  for r, c >= j0, lower tiles only
template <class FC>
__global__ void __launch_bounds__(256) k_ldlt_update(int64_t N, int64_t j0, int64_t jcol, int b, int T,
                                                     FC *__restrict__ F, const double2 *__restrict__ W) {
  __shared__ double2 Ws[16][65];
  __shared__ double2 Ls[16][65];
  int bi, bj;
  lower_tile(blockIdx.x, T, bi, bj);
  int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  int64_t r0 = j0 + (int64_t)bi * 64, c0 = j0 + (int64_t)bj * 64;
  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int jj = 0; jj < 4; jj++) acc[i][jj] = make_double2(0, 0);
  for (int k0 = 0; k0 < b; k0 += 16) {
    for (int e = threadIdx.x; e < 16 * 64; e += 256) {
      int kk = e & 15, rr = e >> 4;
      int64_t r = r0 + rr, cc = c0 + rr;
      bool kin = k0 + kk < b;
      Ws[kk][rr] = (r < N && kin) ? W[r * NB + k0 + kk] : make_double2(0, 0);
      Ls[kk][rr] = (cc < N && kin) ? to_d2(F[cc * N + jcol + k0 + kk]) : make_double2(0, 0);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; kk++) {
      double2 a[4], l[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = Ws[kk][ty + 16 * i];
#pragma unroll
      for (int jj = 0; jj < 4; jj++) l[jj] = Ls[kk][tx + 16 * jj];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int jj = 0; jj < 4; jj++) {
          acc[i][jj].x = fma(a[i].x, l[jj].x, acc[i][jj].x);
          acc[i][jj].x = fma(-a[i].y, l[jj].y, acc[i][jj].x);
          acc[i][jj].y = fma(a[i].x, l[jj].y, acc[i][jj].y);
          acc[i][jj].y = fma(a[i].y, l[jj].x, acc[i][jj].y);
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int jj = 0; jj < 4; jj++) {
      int64_t r = r0 + ty + 16 * i, cc = c0 + tx + 16 * jj;
      if (r < N && cc < N && cc <= r) {
        FC *p = F + r * N + cc;
        store_c(p, csub(to_d2(*p), acc[i][jj]));
      }
    }
}

// inverse of each unit-lower SB x SB diagonal block of L (one CTA per block,
// one thread per column): Linv[blk][i][c]
template <class FC>
__global__ void k_diag_block_inverse(int64_t N, const FC *__restrict__ F, double2 *__restrict__ Linv) {
  // column c of the inverse by forward substitution; the result column is
  // kept in the output buffer itself (L2 resident) instead of registers
  int64_t b0 = (int64_t)blockIdx.x * SB;
  int bs = (int)(N - b0 < SB ? N - b0 : SB);
  int c = threadIdx.x;
  double2 *out = Linv + (int64_t)blockIdx.x * SB * SB;
  if (c >= SB) return;
  for (int i = 0; i < SB; i++) {
    double2 v = make_double2(i == c ? 1.0 : 0.0, 0);
    if (i > c && i < bs) {
      for (int k = c; k < i; k++) v = csub(v, cmul(to_d2(F[(b0 + i) * N + b0 + k]), out[k * SB + c]));
    }
    out[i * SB + c] = (i < c) ? make_double2(0, 0) : v;
  }
}

// ---------------------------------------------------------------------------
// ticket-ordered triangular solves (one RHS column per grid.y)
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool wait_flag(const volatile unsigned *flag, unsigned *err) {
  long long it = 0;
  while (*flag == 0u) {
    if (++it > SPIN_LIMIT) {
      atomicOr(err, 4u);
      return false;
    }
    if (*((volatile unsigned *)err) & 4u) return false;
    __nanosleep(100);
  }
  return true;
}

// forward: L y = x  (x overwritten by y).  flags[rhs][nblk], tickets[rhs]
template <class FC>
__global__ void __launch_bounds__(256) k_trsv_fwd(int64_t N, const FC *__restrict__ F,
                                                  const double2 *__restrict__ Linv, double2 *x,
                                                  unsigned *flags, unsigned *tickets, unsigned *err) {
  __shared__ double2 acc[SB];
  __shared__ double2 part[4][SB];
  __shared__ int s_t;
  int nblk = (int)((N + SB - 1) / SB);
  int rhs = blockIdx.y;
  double2 *xr = x + (int64_t)rhs * N;
  unsigned *fl = flags + (int64_t)rhs * nblk;
  if (threadIdx.x == 0) s_t = (int)atomicAdd(tickets + rhs, 1u);
  __syncthreads();
  int t = s_t;
  int64_t r0 = (int64_t)t * SB;
  int bs = (int)(N - r0 < SB ? N - r0 : SB);
  if (threadIdx.x < SB) acc[threadIdx.x] = threadIdx.x < bs ? xr[r0 + threadIdx.x] : make_double2(0, 0);
  __syncthreads();
  int q = threadIdx.x >> 6, rr = threadIdx.x & 63;
  // block GEMV mapping: 4 row groups x 64 columns, rows reduced across the
  // two warps that share them (coalesced reads of L rows)
  int col = threadIdx.x & 63, rg = threadIdx.x >> 6, half = (threadIdx.x >> 5) & 1;
  for (int cb = 0; cb < t; cb++) {
    if (threadIdx.x == 0) {
      if (!wait_flag(fl + cb, err)) s_t = -1;
    }
    __syncthreads();
    if (s_t < 0) return;
    __threadfence();
    int64_t c0 = (int64_t)cb * SB;
    double2 yv = __ldcg(xr + c0 + col);
    for (int i = 0; i < 16; i++) {
      int row = rg + 4 * i;
      double2 v = make_double2(0, 0);
      if (row < bs) v = cmul(to_d2(F[(r0 + row) * N + c0 + col]), yv);
      v = warp_sum2(v);
      if ((threadIdx.x & 31) == 0) part[half][row] = v;
    }
    __syncthreads();
    if (threadIdx.x < SB) acc[threadIdx.x] = csub(acc[threadIdx.x], cadd(part[0][threadIdx.x], part[1][threadIdx.x]));
    __syncthreads();
  }
  // y_t = Linv_tt acc
  const double2 *Li = Linv + (int64_t)t * SB * SB;
  double2 s = make_double2(0, 0);
  for (int c = q * 16; c < q * 16 + 16; c++) s = cadd(s, cmul(Li[rr * SB + c], acc[c]));
  part[q][rr] = s;
  __syncthreads();
  if (threadIdx.x < bs)
    xr[r0 + threadIdx.x] = cadd(cadd(part[0][threadIdx.x], part[1][threadIdx.x]),
                                cadd(part[2][threadIdx.x], part[3][threadIdx.x]));
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) atomicExch(fl + t, 1u);
}

// backward: L^T x = z  (x overwritten).  Block rows processed bottom-up.
template <class FC>
__global__ void __launch_bounds__(256) k_trsv_bwd(int64_t N, const FC *__restrict__ F,
                                                  const double2 *__restrict__ Linv, double2 *x,
                                                  unsigned *flags, unsigned *tickets, unsigned *err) {
  __shared__ double2 acc[SB];
  __shared__ double2 part[4][SB];
  __shared__ int s_t;
  int nblk = (int)((N + SB - 1) / SB);
  int rhs = blockIdx.y;
  double2 *xr = x + (int64_t)rhs * N;
  unsigned *fl = flags + (int64_t)rhs * nblk;
  if (threadIdx.x == 0) s_t = (int)atomicAdd(tickets + rhs, 1u);
  __syncthreads();
  int t = nblk - 1 - s_t;
  int64_t r0 = (int64_t)t * SB;
  int bs = (int)(N - r0 < SB ? N - r0 : SB);
  if (threadIdx.x < SB) acc[threadIdx.x] = threadIdx.x < bs ? xr[r0 + threadIdx.x] : make_double2(0, 0);
  __syncthreads();
  int q = threadIdx.x >> 6, cc = threadIdx.x & 63;  // 4 row quarters x 64 columns
  for (int cb = nblk - 1; cb > t; cb--) {
    if (threadIdx.x == 0) {
      if (!wait_flag(fl + cb, err)) s_t = -1;
    }
    __syncthreads();
    if (s_t < 0) return;
    __threadfence();
    int64_t c0 = (int64_t)cb * SB;
    int cbs = (int)(N - c0 < SB ? N - c0 : SB);
    double2 s = make_double2(0, 0);
    if (cc < bs) {
      for (int r = q * 16; r < q * 16 + 16; r++) {
        if (r >= cbs) break;
        double2 l = to_d2(F[(c0 + r) * N + r0 + cc]);
        double2 v = __ldcg(xr + c0 + r);
        s = cadd(s, cmul(l, v));
      }
    }
    part[q][cc] = s;
    __syncthreads();
    if (threadIdx.x < SB)
      acc[threadIdx.x] = csub(acc[threadIdx.x], cadd(cadd(part[0][threadIdx.x], part[1][threadIdx.x]),
                                                     cadd(part[2][threadIdx.x], part[3][threadIdx.x])));
    __syncthreads();
  }
  // x_t = Linv_tt^T acc
  const double2 *Li = Linv + (int64_t)t * SB * SB;
  double2 s = make_double2(0, 0);
  for (int r = q * 16; r < q * 16 + 16; r++) s = cadd(s, cmul(Li[r * SB + cc], acc[r]));
  part[q][cc] = s;
  __syncthreads();
  if (threadIdx.x < bs)
    xr[r0 + threadIdx.x] = cadd(cadd(part[0][threadIdx.x], part[1][threadIdx.x]),
                                cadd(part[2][threadIdx.x], part[3][threadIdx.x]));
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) atomicExch(fl + t, 1u);
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

__global__ void k_axpy_sub(int64_t count, const double2 *__restrict__ a, const double2 *__restrict__ b,
                           double2 *__restrict__ out) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) out[i] = csub(a[i], b[i]);
}
__global__ void k_add_inplace(int64_t count, const double2 *__restrict__ a, double2 *__restrict__ x) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) x[i] = cadd(x[i], a[i]);
}

unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

namespace dmb {

void copy_z_out(dmb_ctx *c, double *Z_out) {
  const int64_t N = c->n;
  size_t bytes = sizeof(double2) * N * N;
  if (c->z_prec == DMB_PREC_FP64) {
    DMB_CUDA(cudaMemcpyAsync(Z_out, c->d_Z.p, bytes, cudaMemcpyDeviceToHost, c->stream));
  } else {
    DevBuf tmp;
    tmp.ensure(bytes);
    DMB_LAUNCH(c, k_f2_to_d2, blocks_for(N * N, 256), 256, 0, N * N, c->d_Z.as<float2>(),
               tmp.as<double2>());
    DMB_CUDA(cudaMemcpyAsync(Z_out, tmp.p, bytes, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
  }
  DMB_CUDA(cudaStreamSynchronize(c->stream));
}

void z_entries(dmb_ctx *c, const int64_t *m, const int64_t *n, int64_t count, double *out) {
  if (count == 0) return;
  std::vector<int64_t> mn(2 * count);
  for (int64_t i = 0; i < count; i++) {
    mn[2 * i] = m[i];
    mn[2 * i + 1] = n[i];
  }
  DevBuf dmn, dout;
  dmn.ensure(mn.size() * 8);
  dout.ensure(sizeof(double2) * count);
  DMB_CUDA(cudaMemcpyAsync(dmn.p, mn.data(), mn.size() * 8, cudaMemcpyHostToDevice, c->stream));
  if (c->z_prec == DMB_PREC_FP64)
    DMB_LAUNCH(c, k_entries<double2>, blocks_for(count, 256), 256, 0, count, c->n, dmn.as<int64_t>(),
               c->d_Z.as<double2>(), dout.as<double2>());
  else
    DMB_LAUNCH(c, k_entries<float2>, blocks_for(count, 256), 256, 0, count, c->n, dmn.as<int64_t>(),
               c->d_Z.as<float2>(), dout.as<double2>());
  DMB_CUDA(cudaMemcpyAsync(out, dout.p, sizeof(double2) * count, cudaMemcpyDeviceToHost, c->stream));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
}

void apply_impedance(dmb_ctx *c, const double *zs) {
  DevBuf dz;
  dz.ensure(sizeof(double2) * c->nt);
  DMB_CUDA(cudaMemcpyAsync(dz.p, zs, sizeof(double2) * c->nt, cudaMemcpyHostToDevice, c->stream));
  const TriCache *tc = c->d_tcache.as<TriCache>();
  if (c->z_prec == DMB_PREC_FP64) {
    DMB_LAUNCH(c, k_impedance_offdiag<double2>, blocks_for(c->nt, 128), 128, 0, (int)c->nt, tc, c->nq,
               c->d_wq.as<double>(), dz.as<double2>(), c->n, c->d_Z.as<double2>());
    DMB_LAUNCH(c, k_impedance_diag<double2>, blocks_for(c->n, 128), 128, 0, c->n, tc,
               c->d_rwg_slot.as<int>(), c->nq, c->d_wq.as<double>(), dz.as<double2>(),
               c->d_Z.as<double2>());
  } else {
    DMB_LAUNCH(c, k_impedance_offdiag<float2>, blocks_for(c->nt, 128), 128, 0, (int)c->nt, tc, c->nq,
               c->d_wq.as<double>(), dz.as<double2>(), c->n, c->d_Z.as<float2>());
    DMB_LAUNCH(c, k_impedance_diag<float2>, blocks_for(c->n, 128), 128, 0, c->n, tc,
               c->d_rwg_slot.as<int>(), c->nq, c->d_wq.as<double>(), dz.as<double2>(),
               c->d_Z.as<float2>());
  }
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  c->pc_valid = false;
}

void matvec_dev(dmb_ctx *c, const void *x, void *y, int64_t nrhs) {
  const int64_t N = c->n;
  const double2 *xd = (const double2 *)x;
  double2 *yd = (double2 *)y;
  if (nrhs == 1) {
    unsigned g = blocks_for(N, 8);
    if (c->z_prec == DMB_PREC_FP64)
      DMB_LAUNCH(c, k_gemv<double2>, g, 256, 0, N, c->d_Z.as<double2>(), xd, yd);
    else
      DMB_LAUNCH(c, k_gemv<float2>, g, 256, 0, N, c->d_Z.as<float2>(), xd, yd);
  } else {
    dim3 g(blocks_for(N, 64), blocks_for(nrhs, 64));
    if (c->z_prec == DMB_PREC_FP64)
      DMB_LAUNCH(c, k_gemm_zx<double2>, g, 256, 0, N, nrhs, c->d_Z.as<double2>(), xd, yd);
    else
      DMB_LAUNCH(c, k_gemm_zx<float2>, g, 256, 0, N, nrhs, c->d_Z.as<float2>(), xd, yd);
  }
}

template <class FC> static void ldlt_factor(dmb_ctx *c, FC *F) {
  const int64_t N = c->n;
  c->d_W.ensure(sizeof(double2) * N * NB);
  c->d_flags.ensure(64);
  unsigned *err = c->d_flags.as<unsigned>();
  DMB_CUDA(cudaMemsetAsync(err, 0, 4, c->stream));
  for (int64_t j = 0; j < N; j += NB) {
    int b = (int)std::min<int64_t>(NB, N - j);
    DMB_LAUNCH(c, k_ldlt_diag<FC>, 1, 256, 0, N, j, b, F, err);
    int64_t rest = N - j - b;
    if (rest <= 0) break;
    DMB_LAUNCH(c, k_ldlt_panel<FC>, blocks_for(rest, 8), 256, 0, N, j, b, F, c->d_W.as<double2>());
    int T = (int)((rest + 63) / 64);
    int64_t tiles = (int64_t)T * (T + 1) / 2;
    if (c->kt_enabled) DMB_CUDA(cudaEventRecord(c->kt_ev[0], c->stream));
    DMB_LAUNCH(c, k_ldlt_update<FC>, (unsigned)tiles, 256, 0, N, j + b, j, b, T, F, c->d_W.as<double2>());
    if (c->kt_enabled) {
      DMB_CUDA(cudaEventRecord(c->kt_ev[1], c->stream));
      DMB_CUDA(cudaEventSynchronize(c->kt_ev[1]));
      float ms = 0;
      DMB_CUDA(cudaEventElapsedTime(&ms, c->kt_ev[0], c->kt_ev[1]));
      c->kt_ms += ms;
      c->kt_launches++;
      // algorithmic work: lower triangle (incl. diagonal) x b complex MACs
      c->kt_flops += 8.0 * (double)b * (double)rest * (double)(rest + 1) / 2.0;
    }
  }
  unsigned h_err = 0;
  DMB_CUDA(cudaMemcpyAsync(&h_err, err, 4, cudaMemcpyDeviceToHost, c->stream));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  DMB_REQUIRE(h_err == 0, DMB_ERR_BREAKDOWN,
              "near-field factorisation broke down: zero or non-finite pivot");
  int nblk = (int)((N + SB - 1) / SB);
  c->d_dinv.ensure(sizeof(double2) * (size_t)nblk * SB * SB);
  DMB_LAUNCH(c, k_diag_block_inverse<FC>, nblk, 64, 0, N, F, c->d_dinv.as<double2>());
  DMB_CUDA(cudaStreamSynchronize(c->stream));
}

void nf_build(dmb_ctx *c, double cutoff, int kind) {
  double t0 = now_ms();
  const int64_t N = c->n;
  ensure_cache(c, c->cache_quad_order ? c->cache_quad_order : 3);
  const bool f64 = c->z_prec == DMB_PREC_FP64;
  c->pc_valid = false;
  if (kind == DMB_PRECOND_NF_DIAG) {
    DevBuf tmp;
    tmp.ensure(16);
    DMB_CUDA(cudaMemsetAsync(tmp.p, 0, 16, c->stream));
    c->d_dinv.ensure(sizeof(double2) * N);
    if (f64) {
      DMB_LAUNCH(c, k_diag_max<double2>, 1, 1024, 0, N, c->d_Z.as<double2>(), tmp.as<double>(),
                 (unsigned *)(tmp.as<double>() + 1));
      DMB_LAUNCH(c, k_diag_inv<double2>, blocks_for(N, 256), 256, 0, N, c->d_Z.as<double2>(),
                 tmp.as<double>(), c->d_dinv.as<double2>());
    } else {
      DMB_LAUNCH(c, k_diag_max<float2>, 1, 1024, 0, N, c->d_Z.as<float2>(), tmp.as<double>(),
                 (unsigned *)(tmp.as<double>() + 1));
      DMB_LAUNCH(c, k_diag_inv<float2>, blocks_for(N, 256), 256, 0, N, c->d_Z.as<float2>(),
                 tmp.as<double>(), c->d_dinv.as<double2>());
    }
    double mx[2];
    DMB_CUDA(cudaMemcpyAsync(mx, tmp.p, 16, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
    unsigned bad;
    memcpy(&bad, &mx[1], 4);
    DMB_REQUIRE(bad == 0, DMB_ERR_ARGUMENT, "near-field diagonal entries must be finite");
    DMB_REQUIRE(mx[0] > 0, DMB_ERR_ARGUMENT,
                "cannot build a diagonal preconditioner from an all-zero diagonal");
    c->nnz_ratio = 1.0 / (double)N;
    c->pc_kind = kind;
    c->pc_prec = c->z_prec;
    c->pc_valid = true;
    c->tm.precond_ms = now_ms() - t0;
    return;
  }
  size_t esz = f64 ? sizeof(double2) : sizeof(float2);
  c->d_F.ensure(esz * N * N);
  DevBuf cnt;
  cnt.ensure(8);
  DMB_CUDA(cudaMemsetAsync(cnt.p, 0, 8, c->stream));
  dim3 g(blocks_for(N, 256), (unsigned)N);
  if (f64)
    DMB_LAUNCH(c, (k_nf_mask<double2, double2>), g, 256, 0, N, c->d_Z.as<double2>(),
               c->d_centers.as<double>(), cutoff, c->d_F.as<double2>(), cnt.as<unsigned long long>());
  else
    DMB_LAUNCH(c, (k_nf_mask<float2, float2>), g, 256, 0, N, c->d_Z.as<float2>(),
               c->d_centers.as<double>(), cutoff, c->d_F.as<float2>(), cnt.as<unsigned long long>());
  unsigned long long h_cnt = 0;
  DMB_CUDA(cudaMemcpyAsync(&h_cnt, cnt.p, 8, cudaMemcpyDeviceToHost, c->stream));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  c->nnz_ratio = ((double)h_cnt / (double)N) / (double)N;
  if (f64)
    ldlt_factor(c, c->d_F.as<double2>());
  else
    ldlt_factor(c, c->d_F.as<float2>());
  c->pc_kind = kind;
  c->pc_prec = c->z_prec;
  c->pc_valid = true;
  c->tm.precond_ms = now_ms() - t0;
}

template <class FC> static void ldlt_solve(dmb_ctx *c, const FC *F, double2 *x, int64_t R) {
  const int64_t N = c->n;
  int nblk = (int)((N + SB - 1) / SB);
  size_t flag_words = (size_t)R * nblk + R + 1;
  c->d_flags.ensure(std::max<size_t>(64, 4 * (flag_words + 1)));
  unsigned *err = c->d_flags.as<unsigned>();
  unsigned *tickets = err + 1;
  unsigned *flags = tickets + R;
  const double2 *Linv = c->d_dinv.as<double2>();
  dim3 g(nblk, (unsigned)R);
  DMB_CUDA(cudaMemsetAsync(err, 0, 4 * flag_words + 4, c->stream));
  DMB_LAUNCH(c, k_trsv_fwd<FC>, g, 256, 0, N, F, Linv, x, flags, tickets, err);
  DMB_LAUNCH(c, k_scale_by_dinv<FC>, blocks_for(N * R, 256), 256, 0, N, R, F, x);
  DMB_CUDA(cudaMemsetAsync(tickets, 0, 4 * ((size_t)R * nblk + R), c->stream));
  DMB_LAUNCH(c, k_trsv_bwd<FC>, g, 256, 0, N, F, Linv, x, flags, tickets, err);
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
    if (c->pc_prec == DMB_PREC_FP64)
      ldlt_solve(c, c->d_F.as<double2>(), xd, nrhs);
    else
      ldlt_solve(c, c->d_F.as<float2>(), xd, nrhs);
    return;
  }
  throw DmbError{DMB_ERR_STATE, "preconditioner kind not available"};
}

unsigned read_err_word(dmb_ctx *c) {
  unsigned e = 0;
  DMB_CUDA(cudaMemcpyAsync(&e, c->d_flags.p, 4, cudaMemcpyDeviceToHost, c->stream));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  return e;
}

// solve_forward(:direct): factor Z itself (cutoff = Inf) then refine in FP64:
// x += M^-1 (b - Z x) until the componentwise backward error stalls.
void solve_direct_dev(dmb_ctx *c, const double *b_dev, double *x_dev, int64_t nrhs, double *berr) {
  double t0 = now_ms();
  nf_build(c, INFINITY, DMB_PRECOND_NF_LU);
  const int64_t N = c->n, cnt = N * nrhs;
  DevBuf r, z;
  r.ensure(sizeof(double2) * cnt);
  z.ensure(sizeof(double2) * cnt);
  const double2 *b = (const double2 *)b_dev;
  double2 *x = (double2 *)x_dev;
  DMB_CUDA(cudaMemcpyAsync(x, b, sizeof(double2) * cnt, cudaMemcpyDeviceToDevice, c->stream));
  pc_apply_dev(c, x_dev, nrhs);
  std::vector<double2> hb(cnt), hr(cnt);
  DMB_CUDA(cudaMemcpyAsync(hb.data(), b, sizeof(double2) * cnt, cudaMemcpyDeviceToHost, c->stream));
  double bnorm = 0;
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  for (auto &v : hb) bnorm += v.x * v.x + v.y * v.y;
  bnorm = std::sqrt(bnorm);
  double rel = 0;
  for (int it = 0; it < 6; it++) {
    matvec_dev(c, x, z.p, nrhs);
    DMB_LAUNCH(c, k_axpy_sub, blocks_for(cnt, 256), 256, 0, cnt, b, z.as<double2>(), r.as<double2>());
    DMB_CUDA(cudaMemcpyAsync(hr.data(), r.p, sizeof(double2) * cnt, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
    double rn = 0;
    for (auto &v : hr) rn += v.x * v.x + v.y * v.y;
    rel = bnorm > 0 ? std::sqrt(rn) / bnorm : 0.0;
    if (rel < 1e-14) break;
    pc_apply_dev(c, r.as<double>(), nrhs);
    DMB_LAUNCH(c, k_add_inplace, blocks_for(cnt, 256), 256, 0, cnt, r.as<double2>(), x);
  }
  unsigned e = read_err_word(c);
  DMB_REQUIRE((e & 4u) == 0, DMB_ERR_TIMEOUT, "triangular solve wait expired");
  *berr = rel;
  c->tm.solve_ms = now_ms() - t0;
}

}  // namespace dmb
