// dmb_local.cu -- near-field local-inverse preconditioner and its learned
// correction (no counterpart in the reference; its plain near-field sparse
// preconditioner stays the fallback).
//
// Local inverse.  For every RWG m the nearest <= kmax RWGs whose centres lie
// within `radius` (m included) form S_m; A_m = Z[S_m, S_m] is solved for the
// unit vector of m.  Z is complex symmetric, so the solution is both the row and
// the column of A_m^-1 that belongs to m; the rows form a sparse approximate
// inverse M used as a right preconditioner (Z M y = b, x = M y).
//
// Ring step.  E_m is the larger neighbourhood (radius x2, <= 128, S_m first);
// the ring residual of row z is r = Z[E_m, S_m] z - e_m and its gradient
// g = Z[E_m, S_m]^H r.  One descent step z' = z - eta d with the exact line
// search eta = (B d)^H r / ||B d||^2 (B = Z[E_m, S_m]) never increases ||r||.
// Plain step: d = g.
//
// Learned step.  A small network reads per-neighbour features (relative
// position, block coupling, local-inverse entry, ring gradient) and predicts a
// complex modulation o_j of the direction; the step searches the plane of g
// and g o exactly (2 x 2 least squares on the ring residual), so it is never
// worse than the plain step and reaches the target row when o is ideal
// (d_j = g_j (1 + o_j) with the plain step's eta).  It is trained
// on the GPU by the kernels below toward the least-squares rows
// t = argmin ||Z[E_m, S_m] t - e_m|| (exact local solves the method generates):
// the ideal modulation is o*_j = (z_j - t_j) / (eta g_j) - 1 (clipped), weighted
// by |eta g_j|^2 / |t_m|^2 so the loss measures the row error it removes.
// Network: per neighbour j
//   h_j = tanh(W1 f_j + b1)                  (F -> H)
//   c   = mean_j h_j                          (context)
//   q_j = tanh(W2 [h_j ; c] + b2)            (2H -> H)
//   o_j = W3 q_j + b3                         (H -> 2)
// Loss: mean over rows of sum_j w_j |o_j - o*_j|^2.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>

#include "dmb_device.cuh"
#include "dmb_internal.h"

namespace {

constexpr int NF = 13;            // features per neighbour
constexpr int NH = 32;            // hidden width
constexpr int KS = 64;            // small neighbourhood cap
constexpr int KL = 128;           // large (target) neighbourhood cap
// parameter layout (floats)
constexpr int P_W1 = 0, P_B1 = P_W1 + NH * NF, P_W2 = P_B1 + NH, P_B2 = P_W2 + NH * 2 * NH,
              P_W3 = P_B2 + NH, P_B3 = P_W3 + 2 * NH, P_TOTAL = P_B3 + 2;

unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// ---------------------------------------------------------------------------
// neighbour lists: warp per RWG.  One pass collects the RWGs within `radius`
// (up to NCAND, nearest-first not required) with their squared distances in
// shared memory; a bisection over those candidates finds the distance that
// keeps at most kmax; the RWG itself is stored first.
// ---------------------------------------------------------------------------
constexpr int NCAND = 2048;
constexpr int NB_WARPS = 4;

__global__ void __launch_bounds__(32 * NB_WARPS) k_neighbors(int64_t N, const double *__restrict__ cen, double radius,
                                                             int kmax, int *__restrict__ idx, int *__restrict__ cnt) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int w = threadIdx.x / 32, lane = threadIdx.x & 31;
  int *cid = reinterpret_cast<int *>(smem_raw) + w * NCAND;
  float *cd2 = reinterpret_cast<float *>(smem_raw + sizeof(int) * NCAND * NB_WARPS) + w * NCAND;
  const int64_t m = (int64_t)blockIdx.x * NB_WARPS + w;
  if (m >= N) return;
  const double cx = cen[3 * m], cy = cen[3 * m + 1], cz = cen[3 * m + 2];
  const double r2 = radius * radius;
  int nc = 0;
  for (int64_t base = 0; base < N; base += 32) {
    const int64_t n = base + lane;
    bool take = false;
    float d2f = 0.f;
    if (n < N && n != m) {
      double dx = cen[3 * n] - cx, dy = cen[3 * n + 1] - cy, dz = cen[3 * n + 2] - cz;
      double d2 = dx * dx + dy * dy + dz * dz;
      take = d2 <= r2;
      d2f = (float)d2;
    }
    const unsigned mask = __ballot_sync(0xffffffffu, take);
    const int before = __popc(mask & ((1u << lane) - 1u));
    if (take && nc + before < NCAND) {
      cid[nc + before] = (int)n;
      cd2[nc + before] = d2f;
    }
    nc = min(nc + __popc(mask), NCAND);
  }
  __syncwarp();
  const int room = kmax - 1;  // the RWG itself takes one slot
  float t = (float)r2 * 1.0001f;
  auto count = [&](float th) {
    int c = 0;
    for (int i = lane; i < nc; i += 32) c += cd2[i] <= th;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    return c;
  };
  if (count(t) > room) {
    float lo = 0.f, hi = t;
    for (int it = 0; it < 24; it++) {
      const float mid = 0.5f * (lo + hi);
      if (count(mid) > room) hi = mid;
      else lo = mid;
    }
    t = lo;
  }
  int *out = idx + m * kmax;
  if (lane == 0) out[0] = (int)m;
  int pos = 1;
  for (int base = 0; base < nc; base += 32) {
    const int i = base + lane;
    const bool take = i < nc && cd2[i] <= t;
    const unsigned mask = __ballot_sync(0xffffffffu, take);
    const int before = __popc(mask & ((1u << lane) - 1u));
    if (take && pos + before < kmax) out[pos + before] = cid[i];
    pos += __popc(mask);
  }
  if (lane == 0) cnt[m] = min(pos, kmax);
}

// ---------------------------------------------------------------------------
// local inverse row: one CTA per RWG; A = Z[S,S] (k x k) in shared memory,
// Gaussian elimination with partial pivoting on [A | e_0], back substitution.
// CT is the compute type (float2 / double2); ZC the storage type of Z.
// ---------------------------------------------------------------------------
template <int KM, class CT, class ZC>
__global__ void __launch_bounds__(256) k_local_inverse(int64_t N, const ZC *__restrict__ Z, const int *__restrict__ idx,
                                                       const int *__restrict__ cnt, int kstride,
                                                       double2 *__restrict__ rows, unsigned *__restrict__ err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  CT(*A)[KM + 1] = reinterpret_cast<CT(*)[KM + 1]>(smem_raw);
  CT *rhs = reinterpret_cast<CT *>(smem_raw + sizeof(CT) * KM * (KM + 1));
  __shared__ int sidx[KM];
  __shared__ int piv;
  const int64_t m = blockIdx.x;
  const int k = cnt[m];
  for (int i = threadIdx.x; i < k; i += blockDim.x) sidx[i] = idx[m * kstride + i];
  __syncthreads();
  for (int e = threadIdx.x; e < k * k; e += blockDim.x) {
    int i = e / k, j = e % k;
    double2 z = to_d2(Z[(int64_t)sidx[i] * N + sidx[j]]);
    CT v;
    v.x = z.x;
    v.y = z.y;
    A[i][j] = v;
  }
  for (int i = threadIdx.x; i < k; i += blockDim.x) rhs[i] = (i == 0) ? cone<CT>() : czero<CT>();
  __syncthreads();
  for (int c = 0; c < k; c++) {
    if (threadIdx.x < 32) {
      double best = -1.0;
      int bi = c;
      for (int i = c + threadIdx.x; i < k; i += 32) {
        double a = (double)cabs2(A[i][c]);
        if (a > best) {
          best = a;
          bi = i;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        double ob = __shfl_xor_sync(0xffffffffu, best, o);
        int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      if (threadIdx.x == 0) piv = bi;
    }
    __syncthreads();
    const int p = piv;
    if (p != c) {
      for (int j = threadIdx.x; j < k; j += blockDim.x) {
        CT t = A[c][j];
        A[c][j] = A[p][j];
        A[p][j] = t;
      }
      if (threadIdx.x == 0) {
        CT t = rhs[c];
        rhs[c] = rhs[p];
        rhs[p] = t;
      }
    }
    __syncthreads();
    const CT d = A[c][c];
    if (!((double)cabs2(d) > 0.0)) {
      if (threadIdx.x == 0) atomicOr(err, 16u);
      return;  // uniform
    }
    const CT inv_d = cdiv(cone<CT>(), d);
    const int rest = k - c - 1;
    // eliminate below: row i -= (A[i][c]/d) row c, including the RHS column
    for (int e = threadIdx.x; e < rest * (rest + 1); e += blockDim.x) {
      int i = c + 1 + e / (rest + 1), j = c + 1 + e % (rest + 1);
      CT f = cmul(A[i][c], inv_d);
      if (j < k) A[i][j] = csub(A[i][j], cmul(f, A[c][j]));
      else rhs[i] = csub(rhs[i], cmul(f, rhs[c]));
    }
    __syncthreads();
  }
  // back substitution (one warp, row-parallel reduction)
  if (threadIdx.x < 32) {
    for (int i = k - 1; i >= 0; i--) {
      CT s = czero<CT>();
      for (int j = i + 1 + threadIdx.x; j < k; j += 32) s = cadd(s, cmul(A[i][j], rhs[j]));
      for (int o = 16; o > 0; o >>= 1) {
        s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
        s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
      }
      if (threadIdx.x == 0) rhs[i] = cdiv(csub(rhs[i], s), A[i][i]);
      __syncwarp();
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kstride; i += blockDim.x) {
    double2 v = make_double2(0, 0);
    if (i < k) v = make_double2((double)rhs[i].x, (double)rhs[i].y);
    rows[m * kstride + i] = v;
  }
}

// Least-squares sparse-inverse row on the small support S_m over the rows of
// the extended neighbourhood E_m (both lists start with m):
//   t = argmin_z || Z[E_m, S_m] z - e_m ||_2,   normal equations (B^H B) t = B^H e_m
// B is staged in shared memory (complex64), B^H B accumulated and solved in
// FP64 with partial pivoting.  One CTA per RWG.
template <class ZC>
__global__ void __launch_bounds__(256) k_spai_target(int64_t N, const ZC *__restrict__ Z, const int *__restrict__ idx_s,
                                                     const int *__restrict__ cnt_s, const int *__restrict__ idx_e,
                                                     const int *__restrict__ cnt_e, double2 *__restrict__ tout,
                                                     unsigned *__restrict__ err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2(*G)[KS + 1] = reinterpret_cast<double2(*)[KS + 1]>(smem_raw);
  double2 *rhs = reinterpret_cast<double2 *>(smem_raw + sizeof(double2) * KS * (KS + 1));
  float2(*B)[KS] = reinterpret_cast<float2(*)[KS]>(smem_raw + sizeof(double2) * (KS * (KS + 1) + KS));
  __shared__ int si[KS], ei[KL];
  __shared__ int piv;
  const int64_t m = blockIdx.x;
  const int ks = cnt_s[m], ke = cnt_e[m];
  for (int i = threadIdx.x; i < ks; i += blockDim.x) si[i] = idx_s[m * KS + i];
  for (int i = threadIdx.x; i < ke; i += blockDim.x) ei[i] = idx_e[m * KL + i];
  __syncthreads();
  for (int e = threadIdx.x; e < ke * ks; e += blockDim.x) {
    const int r = e / ks, a = e % ks;
    const double2 z = to_d2(Z[(int64_t)ei[r] * N + si[a]]);
    B[r][a] = make_float2((float)z.x, (float)z.y);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < ks * ks; e += blockDim.x) {
    const int a = e / ks, b = e % ks;
    double2 s = make_double2(0, 0);
    for (int r = 0; r < ke; r++) {
      const float2 x = B[r][a], y = B[r][b];
      s.x += (double)x.x * y.x + (double)x.y * y.y;  // conj(x) * y
      s.y += (double)x.x * y.y - (double)x.y * y.x;
    }
    G[a][b] = s;
  }
  for (int a = threadIdx.x; a < ks; a += blockDim.x) rhs[a] = make_double2(B[0][a].x, -B[0][a].y);  // conj(B[m][a])
  __syncthreads();
  for (int c = 0; c < ks; c++) {
    if (threadIdx.x < 32) {
      double best = -1.0;
      int bi = c;
      for (int i = c + threadIdx.x; i < ks; i += 32) {
        double a = cabs2(G[i][c]);
        if (a > best) {
          best = a;
          bi = i;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        double ob = __shfl_xor_sync(0xffffffffu, best, o);
        int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      if (threadIdx.x == 0) piv = bi;
    }
    __syncthreads();
    const int p = piv;
    if (p != c) {
      for (int j = threadIdx.x; j < ks; j += blockDim.x) {
        double2 t = G[c][j];
        G[c][j] = G[p][j];
        G[p][j] = t;
      }
      if (threadIdx.x == 0) {
        double2 t = rhs[c];
        rhs[c] = rhs[p];
        rhs[p] = t;
      }
    }
    __syncthreads();
    const double2 d = G[c][c];
    if (!(cabs2(d) > 0.0)) {
      if (threadIdx.x == 0) atomicOr(err, 16u);
      return;
    }
    const double2 inv_d = cdiv(make_double2(1, 0), d);
    const int rest = ks - c - 1;
    for (int e = threadIdx.x; e < rest * (rest + 1); e += blockDim.x) {
      int i = c + 1 + e / (rest + 1), j = c + 1 + e % (rest + 1);
      double2 f = cmul(G[i][c], inv_d);
      if (j < ks) G[i][j] = csub(G[i][j], cmul(f, G[c][j]));
      else rhs[i] = csub(rhs[i], cmul(f, rhs[c]));
    }
    __syncthreads();
  }
  if (threadIdx.x < 32) {
    for (int i = ks - 1; i >= 0; i--) {
      double2 s = make_double2(0, 0);
      for (int j = i + 1 + threadIdx.x; j < ks; j += 32) s = cadd(s, cmul(G[i][j], rhs[j]));
      s = warp_sum2(s);
      if (threadIdx.x == 0) rhs[i] = cdiv(csub(rhs[i], s), G[i][i]);
      __syncwarp();
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < KS; i += blockDim.x) tout[m * KS + i] = i < ks ? rhs[i] : make_double2(0, 0);
}

// y[m] = sum_j rows[m][j] x[idx[m][j]] for R right-hand sides
__global__ void k_li_apply(int64_t N, int64_t R, const int *__restrict__ idx, const int *__restrict__ cnt,
                           const double2 *__restrict__ rows, const double2 *__restrict__ x, double2 *__restrict__ y) {
  const int64_t m = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  const int64_t r = blockIdx.y;
  if (m >= N) return;
  const int k = cnt[m];
  double2 s = make_double2(0, 0);
  for (int j = lane; j < k; j += 32) cfma(s, rows[m * KS + j], x[r * N + idx[m * KS + j]]);
  s = warp_sum2(s);
  if (lane == 0) y[r * N + m] = s;
}

// ---------------------------------------------------------------------------
// ring residual of a row: B = Z[E_m, S_m] (E_m: the 2x-radius neighbourhood,
// S_m inside it), r = B z - e_m, g = B^H r (the gradient of ||r||^2 / 2).
// One CTA per RWG.
// ---------------------------------------------------------------------------
template <class ZC>
__global__ void __launch_bounds__(128) k_ring_grad(int64_t N, const ZC *__restrict__ Z, const int *__restrict__ idx_s,
                                                   const int *__restrict__ cnt_s, const int *__restrict__ idx_e,
                                                   const int *__restrict__ cnt_e, const double2 *__restrict__ rows,
                                                   double2 *__restrict__ rring, double2 *__restrict__ grad) {
  __shared__ int si[KS], ei[KL];
  __shared__ double2 z[KS], r[KL];
  const int64_t m = blockIdx.x;
  const int ks = cnt_s[m], ke = cnt_e[m];
  for (int i = threadIdx.x; i < ks; i += blockDim.x) {
    si[i] = idx_s[m * KS + i];
    z[i] = rows[m * KS + i];
  }
  for (int i = threadIdx.x; i < ke; i += blockDim.x) ei[i] = idx_e[m * KL + i];
  __syncthreads();
  for (int e = threadIdx.x; e < KL; e += blockDim.x) {
    double2 s = make_double2(e == 0 ? -1.0 : 0.0, 0.0);
    if (e < ke)
      for (int j = 0; j < ks; j++) cfma(s, to_d2(Z[(int64_t)ei[e] * N + si[j]]), z[j]);
    else
      s = make_double2(0, 0);
    r[e] = s;
    rring[m * KL + e] = s;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < KS; j += blockDim.x) {
    double2 s = make_double2(0, 0);
    if (j < ks)
      for (int e = 0; e < ke; e++) cfma(s, cconj(to_d2(Z[(int64_t)ei[e] * N + si[j]])), r[e]);
    grad[m * KS + j] = s;
  }
}

// One descent step on the ring residual along d_j = g_j (1 + o_j) (o: the
// network's per-entry modulation, or none): exact line search
// eta = (B d)^H r / ||B d||^2, z' = z - eta d.  The ring residual cannot grow.
template <class ZC>
__global__ void __launch_bounds__(128) k_ring_step(int64_t N, const ZC *__restrict__ Z, const int *__restrict__ idx_s,
                                                   const int *__restrict__ cnt_s, const int *__restrict__ idx_e,
                                                   const int *__restrict__ cnt_e, const double2 *__restrict__ rows,
                                                   const double2 *__restrict__ rring, const double2 *__restrict__ grad,
                                                   const float *__restrict__ o, double2 *__restrict__ rows_out,
                                                   double2 *__restrict__ eta_out) {
  __shared__ int si[KS], ei[KL];
  __shared__ double2 d[KS];
  __shared__ double red_n[4][2], red_d[4];
  __shared__ double2 s_eta;
  const int64_t m = blockIdx.x;
  const int ks = cnt_s[m], ke = cnt_e[m];
  for (int i = threadIdx.x; i < ks; i += blockDim.x) {
    si[i] = idx_s[m * KS + i];
    double2 g = grad[m * KS + i];
    if (o) g = cmul(g, make_double2(1.0 + o[(m * KS + i) * 2], o[(m * KS + i) * 2 + 1]));
    d[i] = g;
  }
  for (int i = threadIdx.x; i < ke; i += blockDim.x) ei[i] = idx_e[m * KL + i];
  __syncthreads();
  double nr = 0, ni = 0, dd = 0;
  for (int e = threadIdx.x; e < ke; e += blockDim.x) {
    double2 q = make_double2(0, 0);
    for (int j = 0; j < ks; j++) cfma(q, to_d2(Z[(int64_t)ei[e] * N + si[j]]), d[j]);
    const double2 re = rring[m * KL + e];
    const double2 t = cmul(cconj(q), re);
    nr += t.x;
    ni += t.y;
    dd += cabs2(q);
  }
  nr = warp_sum(nr);
  ni = warp_sum(ni);
  dd = warp_sum(dd);
  if ((threadIdx.x & 31) == 0) {
    red_n[threadIdx.x / 32][0] = nr;
    red_n[threadIdx.x / 32][1] = ni;
    red_d[threadIdx.x / 32] = dd;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0, c = 0;
    for (int w = 0; w < 4; w++) {
      a += red_n[w][0];
      b += red_n[w][1];
      c += red_d[w];
    }
    s_eta = c > 0 ? make_double2(a / c, b / c) : make_double2(0, 0);
    if (eta_out) eta_out[m] = s_eta;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < KS; j += blockDim.x) {
    double2 v = make_double2(0, 0);
    if (j < ks) v = csub(rows[m * KS + j], cmul(s_eta, d[j]));
    rows_out[m * KS + j] = v;
  }
}

// Learned step with a two-direction line search: d1 = g and d2 = g o (the
// network's per-entry modulation); (alpha, beta) minimise the ring residual
// ||r - B (alpha d1 + beta d2)|| exactly (2 x 2 normal equations), so the
// learned step is never worse than the plain step on any row (beta = 0 is
// one of its choices), and with the ideal modulation (alpha = beta = eta) it
// lands on the least-squares row.  A degenerate pair (q2 parallel to q1, or
// zero) falls back to the plain step.
template <class ZC>
__global__ void __launch_bounds__(128) k_ring_step2(int64_t N, const ZC *__restrict__ Z, const int *__restrict__ idx_s,
                                                    const int *__restrict__ cnt_s, const int *__restrict__ idx_e,
                                                    const int *__restrict__ cnt_e, const double2 *__restrict__ rows,
                                                    const double2 *__restrict__ rring, const double2 *__restrict__ grad,
                                                    const float *__restrict__ o, double2 *__restrict__ rows_out) {
  __shared__ int si[KS], ei[KL];
  __shared__ double2 d1[KS], d2[KS];
  __shared__ double red[4][8];
  __shared__ double2 s_ab[2];
  const int64_t m = blockIdx.x;
  const int ks = cnt_s[m], ke = cnt_e[m];
  for (int i = threadIdx.x; i < ks; i += blockDim.x) {
    si[i] = idx_s[m * KS + i];
    const double2 g = grad[m * KS + i];
    d1[i] = g;
    d2[i] = cmul(g, make_double2(o[(m * KS + i) * 2], o[(m * KS + i) * 2 + 1]));
  }
  for (int i = threadIdx.x; i < ke; i += blockDim.x) ei[i] = idx_e[m * KL + i];
  __syncthreads();
  // a11 = |q1|^2, a22 = |q2|^2, a12 = q1^H q2, h1 = q1^H r, h2 = q2^H r
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int e = threadIdx.x; e < ke; e += blockDim.x) {
    double2 q1 = make_double2(0, 0), q2 = make_double2(0, 0);
    for (int j = 0; j < ks; j++) {
      const double2 z = to_d2(Z[(int64_t)ei[e] * N + si[j]]);
      cfma(q1, z, d1[j]);
      cfma(q2, z, d2[j]);
    }
    const double2 re = rring[m * KL + e];
    const double2 a12 = cmul(cconj(q1), q2), h1 = cmul(cconj(q1), re), h2 = cmul(cconj(q2), re);
    acc[0] += cabs2(q1);
    acc[1] += cabs2(q2);
    acc[2] += a12.x;
    acc[3] += a12.y;
    acc[4] += h1.x;
    acc[5] += h1.y;
    acc[6] += h2.x;
    acc[7] += h2.y;
  }
#pragma unroll
  for (int q = 0; q < 8; q++) {
    acc[q] = warp_sum(acc[q]);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32][q] = acc[q];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t[8];
    for (int q = 0; q < 8; q++) t[q] = red[0][q] + red[1][q] + red[2][q] + red[3][q];
    const double a11 = t[0], a22 = t[1];
    const double2 a12 = make_double2(t[2], t[3]), h1 = make_double2(t[4], t[5]), h2 = make_double2(t[6], t[7]);
    const double det = a11 * a22 - cabs2(a12);
    double2 al = make_double2(0, 0), be = make_double2(0, 0);
    if (a11 > 0 && a22 > 0 && det > 1e-10 * a11 * a22) {
      // Cramer: alpha = (a22 h1 - a12 h2) / det, beta = (a11 h2 - conj(a12) h1) / det
      const double2 na = csub(cscale(h1, a22), cmul(a12, h2));
      const double2 nb = csub(cscale(h2, a11), cmul(cconj(a12), h1));
      al = cscale(na, 1.0 / det);
      be = cscale(nb, 1.0 / det);
    } else if (a11 > 0) {
      al = cscale(h1, 1.0 / a11);
    }
    s_ab[0] = al;
    s_ab[1] = be;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < KS; j += blockDim.x) {
    double2 v = make_double2(0, 0);
    if (j < ks) v = csub(csub(rows[m * KS + j], cmul(s_ab[0], d1[j])), cmul(s_ab[1], d2[j]));
    rows_out[m * KS + j] = v;
  }
}

// ---------------------------------------------------------------------------
// network features (per neighbour j of row m):
//   0-2 (c_j - c_m)/r, 3 |c_j - c_m|/r, 4-5 Z[m][j]/Z[m][m], 6-7 z_j/z_m,
//   8 self flag, 9-10 Z[j][j]/Z[m][m], 11-12 g_j / max_j |g_j|
// ---------------------------------------------------------------------------
template <class ZC>
__global__ void k_features(int64_t N, const ZC *__restrict__ Z, const double *__restrict__ cen, double radius,
                           const int *__restrict__ idx, const int *__restrict__ cnt, const double2 *__restrict__ rows,
                           const double2 *__restrict__ grad, float *__restrict__ feat) {
  __shared__ double gmax_w[KS / 32];
  const int64_t m = blockIdx.x;
  const int j = threadIdx.x;  // KS threads
  float *f = feat + (m * KS + j) * NF;
  const int k = cnt[m];
  const double2 gj = j < k ? grad[m * KS + j] : make_double2(0, 0);
  double gm = warp_max(sqrt(cabs2(gj)));
  if ((j & 31) == 0) gmax_w[j / 32] = gm;
  __syncthreads();
  gm = fmax(gmax_w[0], gmax_w[1]);
  if (j >= k) {
    for (int q = 0; q < NF; q++) f[q] = 0.f;
    return;
  }
  const int n = idx[m * KS + j];
  const double2 zmm = to_d2(Z[m * N + m]), zmn = to_d2(Z[m * N + n]), znn = to_d2(Z[(int64_t)n * N + n]);
  const double2 r0 = rows[m * KS], rj = rows[m * KS + j];
  const double2 a = cdiv(zmn, zmm), b = cdiv(znn, zmm), w = cdiv(rj, r0);
  const double inv_r = 1.0 / radius;
  const double dx = (cen[3 * n] - cen[3 * m]) * inv_r, dy = (cen[3 * n + 1] - cen[3 * m + 1]) * inv_r,
               dz = (cen[3 * n + 2] - cen[3 * m + 2]) * inv_r;
  const double ig = gm > 0 ? 1.0 / gm : 0.0;
  f[0] = (float)dx;
  f[1] = (float)dy;
  f[2] = (float)dz;
  f[3] = (float)sqrt(dx * dx + dy * dy + dz * dz);
  f[4] = (float)a.x;
  f[5] = (float)a.y;
  f[6] = (float)w.x;
  f[7] = (float)w.y;
  f[8] = j == 0 ? 1.f : 0.f;
  f[9] = (float)b.x;
  f[10] = (float)b.y;
  f[11] = (float)(gj.x * ig);
  f[12] = (float)(gj.y * ig);
}

// targets for the per-entry step modulation o_j, from the least-squares row t:
//   z_j - eta g_j (1 + o_j) = t_j  =>  o*_j = (z_j - t_j) / (eta g_j) - 1,
// weighted by |eta g_j|^2 / |t_m|^2 so the loss is the row error in z units.
__global__ void k_targets(int64_t N, const int *__restrict__ cnt_s, const double2 *__restrict__ rows_s,
                          const double2 *__restrict__ trow, const double2 *__restrict__ grad,
                          const double2 *__restrict__ eta, float *__restrict__ tgt, float *__restrict__ wgt) {
  const int64_t m = blockIdx.x;
  const int j = threadIdx.x;  // KS threads
  const int ks = cnt_s[m];
  float tr = 0.f, ti = 0.f, w = 0.f;
  if (j < ks) {
    const double2 eg = cmul(eta[m], grad[m * KS + j]);
    const double t0 = cabs2(trow[m * KS]);
    const double eg2 = cabs2(eg);
    if (eg2 > 1e-30 * t0 && t0 > 0) {
      double2 q = csub(cdiv(csub(rows_s[m * KS + j], trow[m * KS + j]), eg), make_double2(1, 0));
      tr = (float)fmin(fmax(q.x, -4.0), 4.0);
      ti = (float)fmin(fmax(q.y, -4.0), 4.0);
      w = (float)(eg2 / t0);
    }
  }
  tgt[(m * KS + j) * 2] = tr;
  tgt[(m * KS + j) * 2 + 1] = ti;
  wgt[m * KS + j] = w;
}

// ---------------------------------------------------------------------------
// network forward / backward (one CTA of KS threads per row)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mlp_forward_row(const float *__restrict__ P, const float *f, int valid, int k,
                                                float *h, float *g, float *out, float *sh_ctx, float *sh_h) {
  // h = tanh(W1 f + b1)
  for (int u = 0; u < NH; u++) {
    float s = P[P_B1 + u];
    for (int q = 0; q < NF; q++) s = fmaf(P[P_W1 + u * NF + q], f[q], s);
    h[u] = valid ? tanhf(s) : 0.f;
    sh_h[threadIdx.x * NH + u] = h[u];
  }
  __syncthreads();
  if (threadIdx.x < NH) {
    float s = 0.f;
    for (int jj = 0; jj < k; jj++) s += sh_h[jj * NH + threadIdx.x];
    sh_ctx[threadIdx.x] = k > 0 ? s / (float)k : 0.f;
  }
  __syncthreads();
  for (int u = 0; u < NH; u++) {
    float s = P[P_B2 + u];
    for (int q = 0; q < NH; q++) s = fmaf(P[P_W2 + u * 2 * NH + q], h[q], s);
    for (int q = 0; q < NH; q++) s = fmaf(P[P_W2 + u * 2 * NH + NH + q], sh_ctx[q], s);
    g[u] = valid ? tanhf(s) : 0.f;
  }
  for (int o = 0; o < 2; o++) {
    float s = P[P_B3 + o];
    for (int q = 0; q < NH; q++) s = fmaf(P[P_W3 + o * NH + q], g[q], s);
    out[o] = valid ? s : 0.f;
  }
}

// inference: per-entry step modulation o[m][j] (2 floats)
__global__ void __launch_bounds__(KS) k_net_infer(int64_t N, const float *__restrict__ P, const float *__restrict__ feat,
                                                  const int *__restrict__ cnt, float *__restrict__ o) {
  __shared__ float sh_h[KS * NH];
  __shared__ float sh_ctx[NH];
  const int64_t m = blockIdx.x;
  const int j = threadIdx.x;
  const int k = cnt[m];
  float f[NF], h[NH], g[NH], out[2];
  for (int q = 0; q < NF; q++) f[q] = feat[(m * KS + j) * NF + q];
  mlp_forward_row(P, f, j < k, k, h, g, out, sh_ctx, sh_h);
  o[(m * KS + j) * 2] = j < k ? out[0] : 0.f;
  o[(m * KS + j) * 2 + 1] = j < k ? out[1] : 0.f;
}

// training: loss and per-row gradient contribution (written to partial[m][P])
__global__ void __launch_bounds__(KS) k_net_grad(int64_t nrows, const int64_t *__restrict__ rowid,
                                                 const float *__restrict__ P, const float *__restrict__ feat,
                                                 const int *__restrict__ cnt, const float *__restrict__ tgt,
                                                 const float *__restrict__ wgt, float *__restrict__ partial,
                                                 float *__restrict__ loss_rows) {
  __shared__ float sh_h[KS * NH];
  __shared__ float sh_ctx[NH];
  __shared__ float sh_dctx[KS * NH];  // per-neighbour contribution to dL/dctx
  __shared__ float sh_grad[P_TOTAL];
  __shared__ float sh_loss[KS];
  const int64_t b = blockIdx.x;
  if (b >= nrows) return;
  const int64_t m = rowid ? rowid[b] : b;
  const int j = threadIdx.x;
  const int k = cnt[m];
  const bool valid = j < k;
  for (int q = threadIdx.x; q < P_TOTAL; q += blockDim.x) sh_grad[q] = 0.f;
  float f[NF], h[NH], g[NH], out[2];
  for (int q = 0; q < NF; q++) f[q] = feat[(m * KS + j) * NF + q];
  mlp_forward_row(P, f, valid, k, h, g, out, sh_ctx, sh_h);
  const float sc = valid ? wgt[m * KS + j] : 0.f;
  float d0 = 0.f, d1 = 0.f, l = 0.f;
  if (valid) {
    const float e0 = out[0] - tgt[(m * KS + j) * 2], e1 = out[1] - tgt[(m * KS + j) * 2 + 1];
    l = sc * (e0 * e0 + e1 * e1);
    d0 = 2.f * sc * e0;
    d1 = 2.f * sc * e1;
  }
  sh_loss[j] = l;
  // backward through layer 3
  float dg[NH];
  for (int q = 0; q < NH; q++) dg[q] = d0 * P[P_W3 + q] + d1 * P[P_W3 + NH + q];
  if (valid) {
    for (int q = 0; q < NH; q++) {
      atomicAdd(&sh_grad[P_W3 + q], d0 * g[q]);
      atomicAdd(&sh_grad[P_W3 + NH + q], d1 * g[q]);
    }
    atomicAdd(&sh_grad[P_B3], d0);
    atomicAdd(&sh_grad[P_B3 + 1], d1);
  }
  // through tanh of layer 2
  float ds[NH];
  for (int u = 0; u < NH; u++) ds[u] = valid ? dg[u] * (1.f - g[u] * g[u]) : 0.f;
  float dh[NH];
  for (int q = 0; q < NH; q++) dh[q] = 0.f;
  for (int q = 0; q < NH; q++) sh_dctx[j * NH + q] = 0.f;
  if (valid) {
    for (int u = 0; u < NH; u++) {
      atomicAdd(&sh_grad[P_B2 + u], ds[u]);
      for (int q = 0; q < NH; q++) {
        atomicAdd(&sh_grad[P_W2 + u * 2 * NH + q], ds[u] * h[q]);
        atomicAdd(&sh_grad[P_W2 + u * 2 * NH + NH + q], ds[u] * sh_ctx[q]);
        dh[q] = fmaf(ds[u], P[P_W2 + u * 2 * NH + q], dh[q]);
        sh_dctx[j * NH + q] = fmaf(ds[u], P[P_W2 + u * 2 * NH + NH + q], sh_dctx[j * NH + q]);
      }
    }
  }
  __syncthreads();
  // context: ctx = mean_j h_j  ->  dh_j += (1/k) sum_i dctx_i
  if (valid) {
    for (int q = 0; q < NH; q++) {
      float s = 0.f;
      for (int i = 0; i < k; i++) s += sh_dctx[i * NH + q];
      dh[q] += s / (float)k;
    }
    // through tanh of layer 1
    for (int u = 0; u < NH; u++) {
      const float da = dh[u] * (1.f - h[u] * h[u]);
      atomicAdd(&sh_grad[P_B1 + u], da);
      for (int q = 0; q < NF; q++) atomicAdd(&sh_grad[P_W1 + u * NF + q], da * f[q]);
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < P_TOTAL; q += blockDim.x) partial[b * P_TOTAL + q] = sh_grad[q];
  if (threadIdx.x == 0) {
    float s = 0.f;
    for (int i = 0; i < KS; i++) s += sh_loss[i];
    loss_rows[b] = s;
  }
}

// grad[p] = sum_b partial[b][p] / nrows; loss = sum_b loss_rows[b] / nrows
__global__ void k_grad_reduce(int64_t nrows, const float *__restrict__ partial, const float *__restrict__ loss_rows,
                              float *__restrict__ grad, float *__restrict__ loss) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < P_TOTAL) {
    double s = 0;
    for (int64_t b = 0; b < nrows; b++) s += partial[b * P_TOTAL + p];
    grad[p] = (float)(s / (double)nrows);
  }
  if (p == P_TOTAL) {
    double s = 0;
    for (int64_t b = 0; b < nrows; b++) s += loss_rows[b];
    *loss = (float)(s / (double)nrows);
  }
}

__global__ void k_adam(float *__restrict__ P, const float *__restrict__ grad, float *__restrict__ m1,
                       float *__restrict__ m2, float lr, float beta1, float beta2, float eps, int step) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P_TOTAL) return;
  const float gr = grad[p];
  m1[p] = beta1 * m1[p] + (1.f - beta1) * gr;
  m2[p] = beta2 * m2[p] + (1.f - beta2) * gr * gr;
  const float mh = m1[p] / (1.f - powf(beta1, (float)step));
  const float vh = m2[p] / (1.f - powf(beta2, (float)step));
  P[p] -= lr * mh / (sqrtf(vh) + eps);
}

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------
struct LocalState {
  DevBuf idx_s, cnt_s, rows_s, idx_l, cnt_l, rows_l, feat, tgt, wgt, partial, lossr, grad, m1, m2, lossv, rowid;
  DevBuf rows_corr, apply_tmp, rring, gring, eta, outs;
  int adam_step = 0;
  double radius = 0;
};

std::mutex g_local_mu;
std::vector<std::pair<dmb_ctx *, LocalState *>> g_local_states;

LocalState &lstate(dmb_ctx *c) {
  std::lock_guard<std::mutex> lk(g_local_mu);
  for (auto &p : g_local_states)
    if (p.first == c) return *p.second;
  g_local_states.push_back({c, new LocalState()});
  return *g_local_states.back().second;
}

template <int KM, class CT> void launch_local_inverse(dmb_ctx *c, const int *idx, const int *cnt, double2 *rows,
                                                      unsigned *err) {
  const size_t sm = sizeof(CT) * (KM * (KM + 1) + KM);
  static bool attr = false;
  if (!attr) {
    if (c->z_prec == DMB_PREC_FP64)
      DMB_CUDA(cudaFuncSetAttribute(k_local_inverse<KM, CT, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)sm));
    DMB_CUDA(cudaFuncSetAttribute(k_local_inverse<KM, CT, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sm));
    DMB_CUDA(cudaFuncSetAttribute(k_local_inverse<KM, CT, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sm));
    attr = true;
  }
  if (c->z_prec == DMB_PREC_FP64)
    DMB_LAUNCH(c, (k_local_inverse<KM, CT, double2>), (unsigned)c->n, 256, sm, c->n, c->d_Z.as<double2>(), idx, cnt,
               KM, rows, err);
  else
    DMB_LAUNCH(c, (k_local_inverse<KM, CT, float2>), (unsigned)c->n, 256, sm, c->n, c->d_Z.as<float2>(), idx, cnt,
               KM, rows, err);
}

void build_neighbors(dmb_ctx *c, double radius, int kmax, DevBuf &idx, DevBuf &cnt) {
  idx.ensure(sizeof(int) * c->n * kmax);
  cnt.ensure(sizeof(int) * c->n);
  const size_t sm = (sizeof(int) + sizeof(float)) * NCAND * NB_WARPS;
  static bool attr = false;
  if (!attr) {
    DMB_CUDA(cudaFuncSetAttribute(k_neighbors, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    attr = true;
  }
  DMB_LAUNCH(c, k_neighbors, blocks_for(c->n, NB_WARPS), 32 * NB_WARPS, sm, c->n, c->d_centers.as<double>(), radius,
             kmax, idx.as<int>(), cnt.as<int>());
}

void ensure_net(dmb_ctx *c, uint64_t seed = 1234) {
  if (c->net_loaded) return;
  std::mt19937_64 rng(seed);
  std::vector<float> p(P_TOTAL, 0.f);
  std::normal_distribution<float> nd(0.f, 1.f);
  for (int i = 0; i < NH * NF; i++) p[P_W1 + i] = nd(rng) * std::sqrt(1.f / NF);
  for (int i = 0; i < NH * 2 * NH; i++) p[P_W2 + i] = nd(rng) * std::sqrt(1.f / (2 * NH));
  for (int i = 0; i < 2 * NH; i++) p[P_W3 + i] = nd(rng) * 0.01f;  // start near the plain local inverse
  c->d_net.ensure(sizeof(float) * P_TOTAL);
  DMB_CUDA(cudaMemcpyAsync(c->d_net.p, p.data(), sizeof(float) * P_TOTAL, cudaMemcpyHostToDevice, c->stream));
  LocalState &st = lstate(c);
  st.m1.ensure(sizeof(float) * P_TOTAL);
  st.m2.ensure(sizeof(float) * P_TOTAL);
  DMB_CUDA(cudaMemsetAsync(st.m1.p, 0, sizeof(float) * P_TOTAL, c->stream));
  DMB_CUDA(cudaMemsetAsync(st.m2.p, 0, sizeof(float) * P_TOTAL, c->stream));
  st.adam_step = 0;
  c->net_loaded = true;
}

void compute_features(dmb_ctx *c, double radius) {
  LocalState &st = lstate(c);
  st.feat.ensure(sizeof(float) * c->n * KS * NF);
  if (c->z_prec == DMB_PREC_FP64)
    DMB_LAUNCH(c, k_features<double2>, (unsigned)c->n, KS, 0, c->n, c->d_Z.as<double2>(), c->d_centers.as<double>(),
               radius, st.idx_s.as<int>(), st.cnt_s.as<int>(), st.rows_s.as<double2>(), st.gring.as<double2>(),
               st.feat.as<float>());
  else
    DMB_LAUNCH(c, k_features<float2>, (unsigned)c->n, KS, 0, c->n, c->d_Z.as<float2>(), c->d_centers.as<double>(),
               radius, st.idx_s.as<int>(), st.cnt_s.as<int>(), st.rows_s.as<double2>(), st.gring.as<double2>(),
               st.feat.as<float>());
}

// ring residual and its gradient for the current rows (needs both neighbour lists)
void ring_grad(dmb_ctx *c) {
  LocalState &st = lstate(c);
  st.rring.ensure(sizeof(double2) * c->n * KL);
  st.gring.ensure(sizeof(double2) * c->n * KS);
  if (c->z_prec == DMB_PREC_FP64)
    DMB_LAUNCH(c, k_ring_grad<double2>, (unsigned)c->n, 128, 0, c->n, c->d_Z.as<double2>(), st.idx_s.as<int>(),
               st.cnt_s.as<int>(), st.idx_l.as<int>(), st.cnt_l.as<int>(), st.rows_s.as<double2>(),
               st.rring.as<double2>(), st.gring.as<double2>());
  else
    DMB_LAUNCH(c, k_ring_grad<float2>, (unsigned)c->n, 128, 0, c->n, c->d_Z.as<float2>(), st.idx_s.as<int>(),
               st.cnt_s.as<int>(), st.idx_l.as<int>(), st.cnt_l.as<int>(), st.rows_s.as<double2>(),
               st.rring.as<double2>(), st.gring.as<double2>());
}

// one line-searched ring step of the rows along g (1 + o); rows_s updated in
// place through rows_corr; eta recorded.  With the network's modulation o the
// step searches the plane of g and g o (k_ring_step2).
void ring_step(dmb_ctx *c, const float *o) {
  LocalState &st = lstate(c);
  st.rows_corr.ensure(sizeof(double2) * c->n * KS);
  st.eta.ensure(sizeof(double2) * c->n);
  if (o) {
    if (c->z_prec == DMB_PREC_FP64)
      DMB_LAUNCH(c, k_ring_step2<double2>, (unsigned)c->n, 128, 0, c->n, c->d_Z.as<double2>(), st.idx_s.as<int>(),
                 st.cnt_s.as<int>(), st.idx_l.as<int>(), st.cnt_l.as<int>(), st.rows_s.as<double2>(),
                 st.rring.as<double2>(), st.gring.as<double2>(), o, st.rows_corr.as<double2>());
    else
      DMB_LAUNCH(c, k_ring_step2<float2>, (unsigned)c->n, 128, 0, c->n, c->d_Z.as<float2>(), st.idx_s.as<int>(),
                 st.cnt_s.as<int>(), st.idx_l.as<int>(), st.cnt_l.as<int>(), st.rows_s.as<double2>(),
                 st.rring.as<double2>(), st.gring.as<double2>(), o, st.rows_corr.as<double2>());
    return;
  }
  if (c->z_prec == DMB_PREC_FP64)
    DMB_LAUNCH(c, k_ring_step<double2>, (unsigned)c->n, 128, 0, c->n, c->d_Z.as<double2>(), st.idx_s.as<int>(),
               st.cnt_s.as<int>(), st.idx_l.as<int>(), st.cnt_l.as<int>(), st.rows_s.as<double2>(),
               st.rring.as<double2>(), st.gring.as<double2>(), o, st.rows_corr.as<double2>(),
               st.eta.as<double2>());
  else
    DMB_LAUNCH(c, k_ring_step<float2>, (unsigned)c->n, 128, 0, c->n, c->d_Z.as<float2>(), st.idx_s.as<int>(),
               st.cnt_s.as<int>(), st.idx_l.as<int>(), st.cnt_l.as<int>(), st.rows_s.as<double2>(),
               st.rring.as<double2>(), st.gring.as<double2>(), o, st.rows_corr.as<double2>(),
               st.eta.as<double2>());
}

void check_err(dmb_ctx *c, const DevBuf &e) {
  unsigned h = 0;
  DMB_CUDA(cudaMemcpyAsync(&h, e.p, 4, cudaMemcpyDeviceToHost, c->stream));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  DMB_REQUIRE(h == 0, DMB_ERR_BREAKDOWN, "local near-field block is singular");
}

}  // namespace

namespace dmb {

// drop the context's local-preconditioner buffers (called when the context is destroyed)
void local_release(dmb_ctx *c) {
  std::lock_guard<std::mutex> lk(g_local_mu);
  for (size_t i = 0; i < g_local_states.size(); i++) {
    if (g_local_states[i].first != c) continue;
    LocalState *st = g_local_states[i].second;
    for (DevBuf *b : {&st->idx_s, &st->cnt_s, &st->rows_s, &st->idx_l, &st->cnt_l, &st->rows_l, &st->feat,
                      &st->tgt, &st->wgt, &st->partial, &st->lossr, &st->grad, &st->m1, &st->m2, &st->lossv,
                      &st->rowid, &st->rows_corr, &st->apply_tmp, &st->rring, &st->gring, &st->eta, &st->outs})
      b->release();
    delete st;
    g_local_states.erase(g_local_states.begin() + i);
    return;
  }
}


// plain local inverses (kind LOCAL_INV) or learned rows (kind LEARNED)
void local_inverse_build(dmb_ctx *c, double radius, int kmax) {
  DMB_REQUIRE(c->z_valid, DMB_ERR_STATE, "no assembled impedance matrix");
  DMB_REQUIRE(radius > 0 && std::isfinite(radius), DMB_ERR_ARGUMENT, "local-inverse radius must be positive");
  DMB_REQUIRE(kmax >= 1 && kmax <= KS, DMB_ERR_ARGUMENT, "local-inverse size must be in 1..64");
  double t0 = now_ms();
  LocalState &st = lstate(c);
  build_neighbors(c, radius, KS, st.idx_s, st.cnt_s);
  st.rows_s.ensure(sizeof(double2) * c->n * KS);
  c->d_small.ensure(65536);
  DevBuf e;
  e.p = c->d_small.p;
  DMB_CUDA(cudaMemsetAsync(e.p, 0, 4, c->stream));
  if (c->z_prec == DMB_PREC_FP64)
    launch_local_inverse<KS, double2>(c, st.idx_s.as<int>(), st.cnt_s.as<int>(), st.rows_s.as<double2>(),
                                      e.as<unsigned>());
  else
    launch_local_inverse<KS, float2>(c, st.idx_s.as<int>(), st.cnt_s.as<int>(), st.rows_s.as<double2>(),
                                     e.as<unsigned>());
  check_err(c, e);
  st.radius = radius;
  c->pc_kind = DMB_PRECOND_LOCAL_INV;
  c->pc_prec = c->z_prec;
  c->pc_valid = true;
  c->nnz_ratio = (double)KS / (double)c->n;
  c->tm.precond_ms = now_ms() - t0;
}

// local inverse, then one line-searched ring step whose per-entry direction is
// modulated by the trained network (learned = true) or not (learned = false)
void ring_step_build(dmb_ctx *c, double radius, bool learned) {
  if (learned) DMB_REQUIRE(c->net_loaded, DMB_ERR_STATE, "no trained network: train or load weights first");
  double t0 = now_ms();
  local_inverse_build(c, radius, KS);
  LocalState &st = lstate(c);
  build_neighbors(c, 2.0 * radius, KL, st.idx_l, st.cnt_l);
  ring_grad(c);
  const float *o = nullptr;
  if (learned) {
    compute_features(c, radius);
    st.outs.ensure(sizeof(float) * c->n * KS * 2);
    DMB_LAUNCH(c, k_net_infer, (unsigned)c->n, KS, 0, c->n, c->d_net.as<float>(), st.feat.as<float>(),
               st.cnt_s.as<int>(), st.outs.as<float>());
    o = st.outs.as<float>();
  }
  ring_step(c, o);
  DMB_CUDA(cudaMemcpyAsync(st.rows_s.p, st.rows_corr.p, sizeof(double2) * c->n * KS, cudaMemcpyDeviceToDevice,
                           c->stream));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  c->pc_kind = learned ? DMB_PRECOND_LEARNED : DMB_PRECOND_RING;
  c->tm.precond_ms = now_ms() - t0;
}

void learned_build(dmb_ctx *c, double radius) { ring_step_build(c, radius, true); }

void local_apply_dev(dmb_ctx *c, double *x, int64_t nrhs) {
  LocalState &st = lstate(c);
  const int64_t N = c->n;
  st.apply_tmp.ensure(sizeof(double2) * N * nrhs);
  double2 *tmp = st.apply_tmp.as<double2>();
  DMB_CUDA(cudaMemcpyAsync(tmp, x, sizeof(double2) * N * nrhs, cudaMemcpyDeviceToDevice, c->stream));
  dim3 g(blocks_for(N, 8), (unsigned)nrhs);
  DMB_LAUNCH(c, k_li_apply, g, 256, 0, N, nrhs, st.idx_s.as<int>(), st.cnt_s.as<int>(), st.rows_s.as<double2>(), tmp,
             (double2 *)x);
}

void ls_rows(dmb_ctx *c, double radius);
double train_epochs(dmb_ctx *c, int epochs, int batch, double lr, uint64_t seed);

// least-squares sparse-inverse rows as the preconditioner (the exact form of
// what the network is trained to approximate); applied like the local inverse
void ls_build(dmb_ctx *c, double radius) {
  double t0 = now_ms();
  local_inverse_build(c, radius, KS);
  ls_rows(c, radius);
  LocalState &st = lstate(c);
  DMB_CUDA(cudaMemcpyAsync(st.rows_s.p, st.rows_l.p, sizeof(double2) * c->n * KS, cudaMemcpyDeviceToDevice,
                           c->stream));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  c->tm.precond_ms = now_ms() - t0;
}

// One training pass over the rows of the current body: plain local inverses
// (radius, <= 64) as the network input, exact inverses of the larger blocks
// (2 x radius, <= 128) as targets, Adam with the given learning rate over
// minibatches of `batch` rows for `epochs` passes.  Returns the mean loss of
// the last pass.
double learned_train_body(dmb_ctx *c, double radius, int epochs, int batch, double lr, uint64_t seed) {
  DMB_REQUIRE(c->z_valid, DMB_ERR_STATE, "no assembled impedance matrix");
  DMB_REQUIRE(epochs >= 1 && batch >= 1, DMB_ERR_ARGUMENT, "epochs and batch must be positive");
  ensure_net(c);
  LocalState &st = lstate(c);
  const int64_t N = c->n;
  // inputs: local inverse rows, their ring gradient, features
  local_inverse_build(c, radius, KS);
  // targets: least-squares sparse-inverse rows over the 2x-radius rows (this
  // also builds the 2x-radius neighbour lists)
  ls_rows(c, radius);
  ring_grad(c);
  compute_features(c, radius);
  ring_step(c, nullptr);  // plain step: eta per row
  st.tgt.ensure(sizeof(float) * N * KS * 2);
  st.wgt.ensure(sizeof(float) * N * KS);
  DMB_LAUNCH(c, k_targets, (unsigned)N, KS, 0, N, st.cnt_s.as<int>(), st.rows_s.as<double2>(),
             st.rows_l.as<double2>(), st.gring.as<double2>(), st.eta.as<double2>(), st.tgt.as<float>(),
             st.wgt.as<float>());
  return train_epochs(c, epochs, batch, lr, seed);
}

// least-squares sparse-inverse rows on the small supports (needs the small
// neighbour lists of local_inverse_build), written to the LocalState rows_l
void ls_rows(dmb_ctx *c, double radius) {
  LocalState &st = lstate(c);
  const int64_t N = c->n;
  build_neighbors(c, 2.0 * radius, KL, st.idx_l, st.cnt_l);
  st.rows_l.ensure(sizeof(double2) * N * KS);
  DevBuf e;
  e.p = c->d_small.p;
  DMB_CUDA(cudaMemsetAsync(e.p, 0, 4, c->stream));
  const size_t sm = sizeof(double2) * (KS * (KS + 1) + KS) + sizeof(float2) * KL * KS;
  static bool attr = false;
  if (!attr) {
    DMB_CUDA(cudaFuncSetAttribute(k_spai_target<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    DMB_CUDA(cudaFuncSetAttribute(k_spai_target<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    attr = true;
  }
  if (c->z_prec == DMB_PREC_FP64)
    DMB_LAUNCH(c, k_spai_target<double2>, (unsigned)N, 256, sm, N, c->d_Z.as<double2>(), st.idx_s.as<int>(),
               st.cnt_s.as<int>(), st.idx_l.as<int>(), st.cnt_l.as<int>(), st.rows_l.as<double2>(), e.as<unsigned>());
  else
    DMB_LAUNCH(c, k_spai_target<float2>, (unsigned)N, 256, sm, N, c->d_Z.as<float2>(), st.idx_s.as<int>(),
               st.cnt_s.as<int>(), st.idx_l.as<int>(), st.cnt_l.as<int>(), st.rows_l.as<double2>(), e.as<unsigned>());
  check_err(c, e);
}

// minibatch Adam over the rows of the current body (features and targets set)
double train_epochs(dmb_ctx *c, int epochs, int batch, double lr, uint64_t seed) {
  LocalState &st = lstate(c);
  const int64_t N = c->n;
  const int64_t B = std::min<int64_t>(batch, N);
  st.partial.ensure(sizeof(float) * B * P_TOTAL);
  st.lossr.ensure(sizeof(float) * B);
  st.grad.ensure(sizeof(float) * P_TOTAL);
  st.lossv.ensure(sizeof(float) * 4);
  st.rowid.ensure(sizeof(int64_t) * N);
  std::mt19937_64 rng(seed);
  std::vector<int64_t> perm(N);
  double last = 0;
  for (int ep = 0; ep < epochs; ep++) {
    for (int64_t i = 0; i < N; i++) perm[i] = i;
    std::shuffle(perm.begin(), perm.end(), rng);
    DMB_CUDA(cudaMemcpyAsync(st.rowid.p, perm.data(), sizeof(int64_t) * N, cudaMemcpyHostToDevice, c->stream));
    double acc = 0;
    int nb = 0;
    for (int64_t b0 = 0; b0 + B <= N; b0 += B) {
      DMB_LAUNCH(c, k_net_grad, (unsigned)B, KS, 0, B, st.rowid.as<int64_t>() + b0, c->d_net.as<float>(),
                 st.feat.as<float>(), st.cnt_s.as<int>(), st.tgt.as<float>(), st.wgt.as<float>(),
                 st.partial.as<float>(), st.lossr.as<float>());
      DMB_LAUNCH(c, k_grad_reduce, blocks_for(P_TOTAL + 1, 128), 128, 0, B, st.partial.as<float>(),
                 st.lossr.as<float>(), st.grad.as<float>(), st.lossv.as<float>());
      st.adam_step++;
      DMB_LAUNCH(c, k_adam, blocks_for(P_TOTAL, 128), 128, 0, c->d_net.as<float>(), st.grad.as<float>(),
                 st.m1.as<float>(), st.m2.as<float>(), (float)lr, 0.9f, 0.999f, 1e-8f, st.adam_step);
      float hl = 0;
      DMB_CUDA(cudaMemcpyAsync(&hl, st.lossv.p, 4, cudaMemcpyDeviceToHost, c->stream));
      DMB_CUDA(cudaStreamSynchronize(c->stream));
      acc += hl;
      nb++;
    }
    last = nb ? acc / nb : 0;
  }
  return last;
}

// loss and gradient for caller-supplied features / targets / per-entry
// weights (gradient check)
void net_loss_grad(dmb_ctx *c, const float *feat, const float *tgt, const float *wgt, const int *cnt,
                   int64_t nrows, float *grad, float *loss) {
  ensure_net(c);
  DevBuf f, t, s, k, part, lr, g, lv;
  f.ensure(sizeof(float) * nrows * KS * NF);
  t.ensure(sizeof(float) * nrows * KS * 2);
  s.ensure(sizeof(float) * nrows * KS);
  k.ensure(sizeof(int) * nrows);
  part.ensure(sizeof(float) * nrows * P_TOTAL);
  lr.ensure(sizeof(float) * nrows);
  g.ensure(sizeof(float) * P_TOTAL);
  lv.ensure(16);
  DMB_CUDA(cudaMemcpyAsync(f.p, feat, sizeof(float) * nrows * KS * NF, cudaMemcpyHostToDevice, c->stream));
  DMB_CUDA(cudaMemcpyAsync(t.p, tgt, sizeof(float) * nrows * KS * 2, cudaMemcpyHostToDevice, c->stream));
  DMB_CUDA(cudaMemcpyAsync(s.p, wgt, sizeof(float) * nrows * KS, cudaMemcpyHostToDevice, c->stream));
  DMB_CUDA(cudaMemcpyAsync(k.p, cnt, sizeof(int) * nrows, cudaMemcpyHostToDevice, c->stream));
  DMB_LAUNCH(c, k_net_grad, (unsigned)nrows, KS, 0, nrows, (const int64_t *)nullptr, c->d_net.as<float>(),
             f.as<float>(), k.as<int>(), t.as<float>(), s.as<float>(), part.as<float>(), lr.as<float>());
  DMB_LAUNCH(c, k_grad_reduce, blocks_for(P_TOTAL + 1, 128), 128, 0, nrows, part.as<float>(), lr.as<float>(),
             g.as<float>(), lv.as<float>());
  DMB_CUDA(cudaMemcpyAsync(grad, g.p, sizeof(float) * P_TOTAL, cudaMemcpyDeviceToHost, c->stream));
  DMB_CUDA(cudaMemcpyAsync(loss, lv.p, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  for (DevBuf *b : {&f, &t, &s, &k, &part, &lr, &g, &lv}) b->release();
}

int net_param_count() { return P_TOTAL; }

void net_set(dmb_ctx *c, const float *w) {
  c->d_net.ensure(sizeof(float) * P_TOTAL);
  DMB_CUDA(cudaMemcpyAsync(c->d_net.p, w, sizeof(float) * P_TOTAL, cudaMemcpyHostToDevice, c->stream));
  if (!c->net_loaded) {
    c->net_loaded = true;
    LocalState &st = lstate(c);
    st.m1.ensure(sizeof(float) * P_TOTAL);
    st.m2.ensure(sizeof(float) * P_TOTAL);
    DMB_CUDA(cudaMemsetAsync(st.m1.p, 0, sizeof(float) * P_TOTAL, c->stream));
    DMB_CUDA(cudaMemsetAsync(st.m2.p, 0, sizeof(float) * P_TOTAL, c->stream));
    st.adam_step = 0;
  }
}

void net_get(dmb_ctx *c, float *w) {
  ensure_net(c);
  DMB_CUDA(cudaMemcpyAsync(w, c->d_net.p, sizeof(float) * P_TOTAL, cudaMemcpyDeviceToHost, c->stream));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
}

}  // namespace dmb
