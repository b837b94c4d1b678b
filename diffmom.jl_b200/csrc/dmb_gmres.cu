// dmb_gmres.cu -- GMRES on the device (solve_gmres, IterativeSolve.jl:341-392).
//
// Semantics follow Krylov.gmres as the reference calls it: x0 = 0, no restart
// (the basis grows up to maxiter vectors), rtol = tol, atol = 0, left
// preconditioning stops on the preconditioned residual estimate
// |g_{j+1}| <= tol * ||M b||, right preconditioning on the true residual
// estimate |g_{j+1}| <= tol * ||b||.  Arnoldi orthogonalisation uses
// classical Gram-Schmidt applied twice (same Krylov basis as Krylov.jl's
// modified Gram-Schmidt up to rounding, two reductions per step instead of
// j+1 sequential ones); Givens rotations and the triangular solve are FP64.
//
// nrhs systems are solved together: every operator application is one Z*X
// product (GEMM) over all still-active columns, while each system keeps its
// own Hessenberg matrix, rotations and stopping test.  When the basis would
// exceed the memory budget the iteration restarts from the current iterate.
#include <algorithm>
#include <cmath>

#include "dmb_device.cuh"
#include "dmb_internal.h"

namespace {

unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// h[r][i] = <V_i(r), w(r)> for i in [0, j]
__global__ void k_dots(int64_t N, int64_t R, int j, int64_t vstride, const double2 *__restrict__ V,
                       const double2 *__restrict__ w, double2 *__restrict__ h, int hld) {
  __shared__ double2 red[32];
  int i = blockIdx.x;
  int64_t r = blockIdx.y;
  const double2 *vi = V + (int64_t)i * vstride + r * N;
  const double2 *wr = w + r * N;
  double re = 0, im = 0;
  for (int64_t n = threadIdx.x; n < N; n += blockDim.x) {
    double2 a = vi[n], b = wr[n];
    re = fma(a.x, b.x, fma(a.y, b.y, re));
    im = fma(a.x, b.y, fma(-a.y, b.x, im));
  }
  double2 v = warp_sum2(make_double2(re, im));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : make_double2(0, 0);
    v = warp_sum2(v);
    if (threadIdx.x == 0) h[r * hld + i] = v;
  }
  (void)j;
}

// w(r) -= sum_i h[r][i] V_i(r); H[r][:, j] += h
__global__ void k_cgs_update(int64_t N, int64_t R, int j, int64_t vstride, const double2 *__restrict__ V,
                             const double2 *__restrict__ h, int hld, double2 *__restrict__ w) {
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= N * R) return;
  int64_t r = idx / N, n = idx % N;
  double2 acc = w[idx];
  for (int i = 0; i <= j; i++) acc = csub(acc, cmul(h[r * hld + i], V[(int64_t)i * vstride + r * N + n]));
  w[idx] = acc;
}

__global__ void k_hacc(int64_t R, int j, const double2 *__restrict__ h, int hld, double2 *__restrict__ H,
                       int kcap) {
  int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  double2 *Hr = H + r * (int64_t)(kcap + 1) * kcap + (int64_t)j * (kcap + 1);
  for (int i = 0; i <= j; i++) Hr[i] = cadd(Hr[i], h[r * hld + i]);
}

__global__ void k_norms(int64_t N, const double2 *__restrict__ w, double *__restrict__ out) {
  __shared__ double red[32];
  int64_t r = blockIdx.x;
  const double2 *wr = w + r * N;
  double s = 0;
  for (int64_t n = threadIdx.x; n < N; n += blockDim.x) s += cabs2(wr[n]);
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : 0;
    s = warp_sum(s);
    if (threadIdx.x == 0) out[r] = sqrt(s);
  }
}

__global__ void k_scale_cols(int64_t N, int64_t R, const double *__restrict__ nrm, const double2 *__restrict__ w,
                             double2 *__restrict__ out) {
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= N * R) return;
  double d = nrm[idx / N];
  out[idx] = d > 0 ? cscale(w[idx], 1.0 / d) : make_double2(0, 0);
}

struct SysState {
  double beta;     // ||r0||
  double eps;      // stopping threshold
  double resid;    // |g_k|: the estimate at the solution's basis size k
  double resid_x;  // |g_kx|: the estimate with every processed column
  int k;           // basis size of the solution (iterations)
  int kx;          // Hessenberg columns processed (>= k: a converged system
                   // keeps being rotated while others iterate, so it can be
                   // reactivated without losing its Krylov space)
  int done;        // 1 converged, 2 breakdown/zero rhs, 3 non-finite
  int pad;
};

// start: g = (beta, 0, ...); thresholds
__global__ void k_init_state(int64_t R, const double *__restrict__ nrm, double tol, SysState *__restrict__ st,
                             double2 *__restrict__ g, int kcap) {
  int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  SysState s;
  s.beta = nrm[r];
  s.eps = tol * nrm[r];
  s.resid = nrm[r];
  s.resid_x = nrm[r];
  s.k = 0;
  s.kx = 0;
  s.pad = 0;
  s.done = nrm[r] == 0.0 ? 2 : 0;
  st[r] = s;
  double2 *gr = g + r * (int64_t)(kcap + 1);
  for (int i = 0; i <= kcap; i++) gr[i] = make_double2(0, 0);
  gr[0] = make_double2(nrm[r], 0);
}

// Givens update of column j for every active system
__global__ void k_givens(int64_t R, int j, int kcap, double2 *__restrict__ H, const double *__restrict__ hnext,
                         double *__restrict__ cs, double2 *__restrict__ sn, double2 *__restrict__ g,
                         SysState *__restrict__ st, unsigned *__restrict__ active) {
  int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  SysState s = st[r];
  if (s.done >= 2) return;
  double2 *Hc = H + r * (int64_t)(kcap + 1) * kcap + (int64_t)j * (kcap + 1);
  double *c = cs + r * (int64_t)kcap;
  double2 *sv = sn + r * (int64_t)kcap;
  double2 *gr = g + r * (int64_t)(kcap + 1);
  Hc[j + 1] = make_double2(hnext[r], 0);
  // previous rotations: [c s; -conj(s) c]
  for (int i = 0; i < j; i++) {
    double2 a = Hc[i], b = Hc[i + 1];
    Hc[i] = cadd(cscale(a, c[i]), cmul(sv[i], b));
    Hc[i + 1] = csub(cscale(b, c[i]), cmul(cconj(sv[i]), a));
  }
  double2 a = Hc[j], b = Hc[j + 1];
  double na = hypot(a.x, a.y), nb = hypot(b.x, b.y);
  double cc;
  double2 ss, rho;
  if (nb == 0.0) {
    cc = 1.0; ss = make_double2(0, 0); rho = a;
  } else if (na == 0.0) {
    cc = 0.0; ss = cdiv(cconj(b), make_double2(nb, 0)); rho = make_double2(nb, 0);
  } else {
    double t = hypot(na, nb);
    double2 sa = cscale(a, 1.0 / na);
    cc = na / t;
    ss = cscale(cmul(sa, cconj(b)), 1.0 / t);
    rho = cscale(sa, t);
  }
  c[j] = cc;
  sv[j] = ss;
  Hc[j] = rho;
  Hc[j + 1] = make_double2(0, 0);
  double2 gj = gr[j];
  gr[j] = cscale(gj, cc);
  gr[j + 1] = cscale(cmul(cconj(ss), gj), -1.0);
  s.kx = j + 1;
  s.resid_x = hypot(gr[j + 1].x, gr[j + 1].y);
  if (s.done == 0) {
    s.k = j + 1;
    s.resid = s.resid_x;
    if (s.resid <= s.eps) s.done = 1;
    else if (hnext[r] == 0.0) s.done = 2;  // lucky breakdown: exact solution in the space
    if (!isfinite(s.resid)) s.done = 3;
  }
  st[r] = s;
  if (!s.done) atomicAdd(active, 1u);
}

// y = R^-1 g (back substitution, per system), stored in y[r][i]
__global__ void k_backsolve(int64_t R, int kcap, const double2 *__restrict__ H, const double2 *__restrict__ g,
                            const SysState *__restrict__ st, double2 *__restrict__ y) {
  int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  int k = st[r].k;
  const double2 *Hr = H + r * (int64_t)(kcap + 1) * kcap;
  const double2 *gr = g + r * (int64_t)(kcap + 1);
  double2 *yr = y + r * (int64_t)kcap;
  for (int i = k - 1; i >= 0; i--) {
    double2 v = gr[i];
    for (int l = i + 1; l < k; l++) v = csub(v, cmul(Hr[(int64_t)l * (kcap + 1) + i], yr[l]));
    double2 d = Hr[(int64_t)i * (kcap + 1) + i];
    yr[i] = (d.x == 0 && d.y == 0) ? make_double2(0, 0) : cdiv(v, d);
  }
  for (int i = k; i < kcap; i++) yr[i] = make_double2(0, 0);
}

// x(r) += sum_i y[r][i] V_i(r)
__global__ void k_combine(int64_t N, int64_t R, int kmax, int64_t vstride, const double2 *__restrict__ V,
                          const double2 *__restrict__ y, int kcap, double2 *__restrict__ x) {
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= N * R) return;
  int64_t r = idx / N, n = idx % N;
  double2 acc = make_double2(0, 0);
  for (int i = 0; i < kmax; i++) acc = cadd(acc, cmul(y[r * kcap + i], V[(int64_t)i * vstride + r * N + n]));
  x[idx] = cadd(x[idx], acc);
}

// r = b - sum_i y[r][i] W_i(r): the residual of x = sum_i y_i z_i from the
// stored products W_i = Z z_i
__global__ void k_resid_products(int64_t N, int64_t R, int kmax, int64_t vstride, const double2 *__restrict__ W,
                                 const double2 *__restrict__ y, int kcap, const double2 *__restrict__ b,
                                 double2 *__restrict__ out) {
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= N * R) return;
  int64_t r = idx / N, n = idx % N;
  double2 acc = make_double2(0, 0);
  for (int i = 0; i < kmax; i++) acc = cadd(acc, cmul(y[r * kcap + i], W[(int64_t)i * vstride + r * N + n]));
  out[idx] = csub(b[idx], acc);
}

__global__ void k_sub(int64_t count, const double2 *__restrict__ a, double2 *__restrict__ b) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) b[i] = csub(a[i], b[i]);
}

}  // namespace

namespace dmb {

// w = op(v).  Right preconditioning keeps z = M^-1 v (flexible GMRES form):
// the solution is then sum y_i z_i and needs no further preconditioner
// application, and an inexact (tensor-core) preconditioner stays consistent.
void apply_operator(dmb_ctx *c, int precond_kind, int side, const double2 *v, double2 *w, double2 *z,
                    int64_t R, bool full_levels = false) {
  const int64_t N = c->n;
  if (precond_kind == DMB_PRECOND_NONE) {
    matvec_op(c, v, w, R, full_levels);
  } else if (side == DMB_SIDE_LEFT) {
    matvec_op(c, v, w, R, full_levels);
    pc_apply_dev(c, (double *)w, R);
  } else {
    DMB_CUDA(cudaMemcpyAsync(z, v, sizeof(double2) * N * R, cudaMemcpyDeviceToDevice, c->stream));
    pc_apply_dev(c, (double *)z, R);
    matvec_op(c, z, w, R, full_levels);
  }
}

unsigned read_err_word(dmb_ctx *c);

void gmres_dev(dmb_ctx *c, const double *b_dev, double *x_dev, int64_t R, double tol, int maxiter,
               int precond_kind, int side, dmb_gmres_stats *out) {
  double t0 = now_ms();
  const int64_t N = c->n;
  if (precond_kind != DMB_PRECOND_NONE)
    DMB_REQUIRE(c->pc_valid, DMB_ERR_STATE, "preconditioner requested but not built");
  DMB_REQUIRE(precond_kind == DMB_PRECOND_NONE || precond_kind == c->pc_kind, DMB_ERR_STATE,
              "requested preconditioner kind differs from the one built");
  // basis capacity: maxiter vectors, bounded by a 40% share of free memory
  // (decided once per problem shape; repeated solves reuse the buffers); the
  // right-preconditioned form also keeps the preconditioned vectors
  const bool flex = precond_kind != DMB_PRECOND_NONE && side == DMB_SIDE_RIGHT;
  // With the INT8-slice operator and no left preconditioner, the Krylov
  // products are Z z_i themselves: computed with every slice level (FP64-
  // accurate) and kept before orthogonalisation, they give the true residual
  // of x = sum y_i z_i as b - sum y_i Z z_i without another product.
  const bool prod_resid = krylov_exact_int8(c, R) && (precond_kind == DMB_PRECOND_NONE || side == DMB_SIDE_RIGHT);
  const int nvec = (flex ? 2 : 1) + (prod_resid ? 1 : 0);
  size_t vec_bytes = sizeof(double2) * N * R;
  if (!(c->gm_key_n == N && c->gm_key_r == R && c->gm_key_maxiter == maxiter && c->gm_key_flex == flex &&
        c->gm_key_nvec == nvec && c->gm_kcap > 0)) {
    size_t freeb = 0, totb = 0;
    DMB_CUDA(cudaMemGetInfo(&freeb, &totb));
    freeb += c->d_V.bytes + c->d_Zv.bytes;  // the current buffers can be reused
    // many right-hand sides: at most 8 GiB of basis (a strong preconditioner
    // needs a handful of vectors; GMRES restarts if the capacity runs out)
    double budget = freeb * 0.4;
    if (R >= 8) budget = std::min(budget, 8.0 * 1024 * 1024 * 1024);
    int64_t cap_mem = (int64_t)(budget / (double)(vec_bytes * nvec)) - 1;
    c->gm_kcap = (int)std::max<int64_t>(2, std::min<int64_t>(maxiter, cap_mem));
    c->gm_key_n = N;
    c->gm_key_r = R;
    c->gm_key_maxiter = maxiter;
    c->gm_key_flex = flex;
    c->gm_key_nvec = nvec;
  }
  const int kcap = c->gm_kcap;
  const int64_t vstride = N * R;
  c->d_V.ensure(vec_bytes * (kcap + 1));
  if (flex) c->d_Zv.ensure(vec_bytes * kcap);
  double2 *Zv = flex ? c->d_Zv.as<double2>() : nullptr;
  if (prod_resid) c->d_Wraw.ensure(vec_bytes * kcap);
  double2 *Wraw = prod_resid ? c->d_Wraw.as<double2>() : nullptr;
  c->d_work.ensure(vec_bytes * 2);
  // layout: H[R][(k+1)k] g[R][k+1] sn[R][k] hb[R][k+1] y[R][k] | cs[R][k] nrm[2R] | st[R] | active
  size_t small = sizeof(double2) * R * ((size_t)(kcap + 1) * kcap + 2 * (kcap + 1) + 2 * kcap) +
                 sizeof(double) * R * (kcap + 3) + sizeof(SysState) * R + 64;
  c->d_H.ensure(small);
  double2 *V = c->d_V.as<double2>();
  double2 *w = c->d_work.as<double2>();
  double2 *tmp = w + N * R;
  double2 *H = c->d_H.as<double2>();
  double2 *g = H + R * (int64_t)(kcap + 1) * kcap;
  double2 *sn = g + R * (int64_t)(kcap + 1);
  double2 *hb = sn + R * (int64_t)kcap;
  double2 *ybuf = hb + R * (int64_t)(kcap + 1);
  double *cs = (double *)(ybuf + R * (int64_t)kcap);
  double *nrm = cs + R * (int64_t)kcap;   // [0,R) Krylov norms, [R,2R) ||b||, [2R,3R) ||b - Z x||
  double *tnrm = nrm + 2 * R;
  SysState *st = (SysState *)(nrm + 3 * R);
  unsigned *active = (unsigned *)(st + R);
  const double2 *b = (const double2 *)b_dev;
  double2 *x = (double2 *)x_dev;

  // With the tensor-core operator (FP32 accumulation) the Krylov recurrence
  // is only as exact as that product: a system whose estimate converged is
  // re-checked against the residual computed in FP64 and, if that is still
  // above its threshold, refined by another cycle from the current x.
  const bool inexact = matvec_op_inexact(c, R);
  // few systems with a cheap preconditioner (none, Jacobi, sparse local rows):
  // iterations are short, so host round trips are amortised over several;
  // otherwise an iteration (many systems, or triangular solves) costs far more
  // than the round trip and every one is checked
  const bool cheap = precond_kind != DMB_PRECOND_NF_LU;
  const int check_every = (R < 32 && cheap) ? 4 : 1;
  int iters_used = 0;
  DMB_CUDA(cudaMemsetAsync(x, 0, vec_bytes, c->stream));
  int total_iters = 0, restarts = 0, cycles = 0, j_last = 0;
  bool first = true, have_true = false;
  std::vector<SysState> hst(R);
  // check passes: per system, the factor by which the next cycle must reduce
  // its starting (preconditioned, for left) residual; 0 = keep the threshold
  std::vector<double> recheck_scale(R, 0.0);
  // left preconditioning without an inexact operator: the check continues the
  // cycle instead of restarting it
  const bool left_recheck = c->true_residual_check && precond_kind != DMB_PRECOND_NONE && side == DMB_SIDE_LEFT &&
                            !inexact;
  int recheck_continuations = 0;
  std::vector<double> hn_final(2 * R);
  for (int check_pass = 0;; check_pass++) {
  while (true) {
    // r0 = b - Z x (x = 0 on the first cycle), preconditioned on the left
    if (first) {
      DMB_CUDA(cudaMemcpyAsync(V, b, vec_bytes, cudaMemcpyDeviceToDevice, c->stream));
    } else {
      matvec_dev(c, x, V, R);
      DMB_LAUNCH(c, k_sub, blocks_for(N * R, 256), 256, 0, N * R, b, V);
      if (inexact) DMB_LAUNCH(c, k_norms, (unsigned)R, 256, 0, N, V, tnrm);
    }
    if (precond_kind != DMB_PRECOND_NONE && side == DMB_SIDE_LEFT) pc_apply_dev(c, (double *)V, R);
    DMB_LAUNCH(c, k_norms, (unsigned)R, 256, 0, N, V, nrm);
    if (first) {
      DMB_LAUNCH(c, k_init_state, blocks_for(R, 128), 128, 0, R, nrm, tol, st, g, kcap);
    } else {
      // restart or refinement: keep each system's original threshold
      std::vector<double> hn(R);
      DMB_CUDA(cudaMemcpyAsync(hn.data(), nrm, 8 * R, cudaMemcpyDeviceToHost, c->stream));
      DMB_CUDA(cudaStreamSynchronize(c->stream));
      std::vector<double2> hg((size_t)R * (kcap + 1), make_double2(0, 0));
      bool any = false;
      for (int64_t r = 0; r < R; r++) {
        hst[r].k = 0;
        hst[r].kx = 0;
        hst[r].resid = hn[r];
        hst[r].resid_x = hn[r];
        if (recheck_scale[r] > 0) {
          hst[r].eps = hn[r] * recheck_scale[r];
          recheck_scale[r] = 0;
        }
        if (inexact && hst[r].done == 1 && !(hn[r] <= hst[r].eps)) hst[r].done = 0;
        if (!hst[r].done) {
          hg[(size_t)r * (kcap + 1)] = make_double2(hn[r], 0);
          any = true;
        }
      }
      if (!any) {
        have_true = inexact;  // x has not changed since tnrm was formed
        break;
      }
      if (total_iters >= maxiter) break;
      restarts++;
      DMB_CUDA(cudaMemcpyAsync(st, hst.data(), sizeof(SysState) * R, cudaMemcpyHostToDevice, c->stream));
      DMB_CUDA(cudaMemcpyAsync(g, hg.data(), sizeof(double2) * hg.size(), cudaMemcpyHostToDevice, c->stream));
    }
    first = false;
    cycles++;
    DMB_CUDA(cudaMemsetAsync(H, 0, sizeof(double2) * R * (int64_t)(kcap + 1) * kcap, c->stream));
    DMB_LAUNCH(c, k_scale_cols, blocks_for(N * R, 256), 256, 0, N, R, nrm, V, V);
    // few right-hand sides: iterations between host checks are launch-bound
    // enough to replay as graphs (kernel timing records events per launch)
    const bool graphs_ok = R < 32 && !c->kt_enabled;
    // one Arnoldi + Givens iteration (device work only)
    auto iteration = [&](int jj) {
      double2 *Vj = V + (int64_t)jj * vstride;
      apply_operator(c, precond_kind, side, Vj, w, flex ? Zv + (int64_t)jj * vstride : tmp, R, prod_resid);
      if (prod_resid)
        DMB_CUDA(cudaMemcpyAsync(Wraw + (int64_t)jj * vstride, w, vec_bytes, cudaMemcpyDeviceToDevice, c->stream));
      for (int pass = 0; pass < 2; pass++) {
        DMB_LAUNCH(c, k_dots, dim3(jj + 1, (unsigned)R), 256, 0, N, R, jj, vstride, V, w, hb, kcap + 1);
        DMB_LAUNCH(c, k_cgs_update, blocks_for(N * R, 256), 256, 0, N, R, jj, vstride, V, hb, kcap + 1, w);
        DMB_LAUNCH(c, k_hacc, blocks_for(R, 128), 128, 0, R, jj, hb, kcap + 1, H, kcap);
      }
      DMB_LAUNCH(c, k_norms, (unsigned)R, 256, 0, N, w, nrm);
      DMB_LAUNCH(c, k_scale_cols, blocks_for(N * R, 256), 256, 0, N, R, nrm, w, V + (int64_t)(jj + 1) * vstride);
      DMB_CUDA(cudaMemsetAsync(active, 0, 4, c->stream));
      DMB_LAUNCH(c, k_givens, blocks_for(R, 128), 128, 0, R, jj, kcap, H, nrm, cs, sn, g, st, active);
    };
    // iterations j0 .. j0 + nb - 1, directly or as a captured graph
    auto run_block = [&](int j0, int nb) {
      auto eager = [&] {
        for (int jj = j0; jj < j0 + nb; jj++) iteration(jj);
      };
      if (!(graphs_ok && c->gmres_graphs)) return eager();
      const std::vector<int64_t> key = {j0, nb, N, R, kcap, vstride, precond_kind, side, flex, c->pc_kind,
                                        c->z_prec, (int64_t)(uintptr_t)V, (int64_t)(uintptr_t)Zv,
                                        (int64_t)(uintptr_t)w, (int64_t)(uintptr_t)tmp, (int64_t)(uintptr_t)H,
                                        (int64_t)(uintptr_t)hb, (int64_t)(uintptr_t)g,
                                        (int64_t)(uintptr_t)st, (int64_t)g_dev_alloc_epoch.load()};
      dmb_ctx::GraphEntry &e = c->gm_graphs[key];
      if (e.exec) {
        DMB_CUDA(cudaGraphLaunch(e.exec, c->stream));
        c->launches += e.kernels;
        return;
      }
      if (!e.seen) {  // first meeting: direct launches (any lazy allocation happens here)
        e.seen = true;
        return eager();
      }
      const int64_t l0 = c->launches;
      int64_t kernels = 0;
      cudaGraph_t graph = nullptr;
      bool captured = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      if (captured) {
        try {
          eager();
        } catch (...) {
          captured = false;
        }
        kernels = c->launches - l0;
        cudaGraph_t got = nullptr;
        const bool ended = cudaStreamEndCapture(c->stream, &got) == cudaSuccess;
        if (captured && ended && got) graph = got;
        else if (got) cudaGraphDestroy(got);
      }
      c->launches = l0;  // captured launches have not run
      cudaGraphExec_t ex = nullptr;
      if (graph && cudaGraphInstantiate(&ex, graph, 0) != cudaSuccess) ex = nullptr;
      if (graph) cudaGraphDestroy(graph);
      if (!ex) {  // capture not possible here: direct launches from now on
        (void)cudaGetLastError();
        c->gmres_graphs = false;
        return eager();
      }
      e.exec = ex;
      e.kernels = kernels;  // kernels of one replay: the launches of one direct pass
      DMB_CUDA(cudaGraphLaunch(ex, c->stream));
      c->launches += kernels;
    };
    int j = 0;
    while (j < kcap && total_iters < maxiter) {
      // the iterations up to the next host look at the active count (a system
      // that converged in between keeps its own k; its extra basis vectors
      // are never combined)
      int nb = 1;
      while (j + nb < kcap && total_iters + nb < maxiter && (j + nb) % check_every != 0) nb++;
      run_block(j, nb);
      j += nb;
      total_iters += nb;
      unsigned h_active = 0;
      DMB_CUDA(cudaMemcpyAsync(&h_active, active, 4, cudaMemcpyDeviceToHost, c->stream));
      DMB_CUDA(cudaStreamSynchronize(c->stream));
      // Left preconditioning stops on the preconditioned residual.  With the
      // check on, the trial solution of this cycle is checked against the
      // unpreconditioned FP64 residual; a system that fails it continues the
      // same Arnoldi process (its Krylov space kept) with its threshold
      // lowered by the factor the true residual still needs, margin 2.
      while (h_active == 0 && left_recheck) {
        DMB_LAUNCH(c, k_backsolve, blocks_for(R, 128), 128, 0, R, kcap, H, g, st, ybuf);
        DMB_CUDA(cudaMemcpyAsync(tmp, x, vec_bytes, cudaMemcpyDeviceToDevice, c->stream));
        DMB_LAUNCH(c, k_combine, blocks_for(N * R, 256), 256, 0, N, R, j, vstride, V, ybuf, kcap, tmp);
        matvec_dev(c, tmp, w, R);
        DMB_LAUNCH(c, k_sub, blocks_for(N * R, 256), 256, 0, N * R, b, w);
        DMB_LAUNCH(c, k_norms, (unsigned)R, 256, 0, N, w, tnrm);
        DMB_LAUNCH(c, k_norms, (unsigned)R, 256, 0, N, b, nrm + R);
        std::vector<double> hr(2 * R);
        DMB_CUDA(cudaMemcpyAsync(hr.data(), nrm + R, 16 * R, cudaMemcpyDeviceToHost, c->stream));
        DMB_CUDA(cudaMemcpyAsync(hst.data(), st, sizeof(SysState) * R, cudaMemcpyDeviceToHost, c->stream));
        DMB_CUDA(cudaStreamSynchronize(c->stream));
        bool changed = false;
        for (int64_t r = 0; r < R; r++) {
          const double bn = hr[r], rn = hr[R + r];
          SysState &sr = hst[r];
          if (sr.done != 1 || !(bn > 0) || !std::isfinite(rn) || rn <= tol * bn) continue;
          const double eps_new = sr.resid * std::min(0.5, 0.5 * tol * bn / rn);
          if (sr.resid_x <= eps_new) {  // the columns processed since already suffice
            if (sr.kx == sr.k) continue;
            sr.k = sr.kx;
            sr.resid = sr.resid_x;
          } else {
            sr.done = 0;
            sr.k = sr.kx;
            sr.resid = sr.resid_x;
            h_active++;
          }
          sr.eps = eps_new;
          changed = true;
        }
        if (!changed) break;
        recheck_continuations++;
        DMB_CUDA(cudaMemcpyAsync(st, hst.data(), sizeof(SysState) * R, cudaMemcpyHostToDevice, c->stream));
      }
      if (h_active == 0) break;
    }
    // solution update from this cycle
    j_last = j;
    DMB_LAUNCH(c, k_backsolve, blocks_for(R, 128), 128, 0, R, kcap, H, g, st, ybuf);
    if (flex) {
      DMB_LAUNCH(c, k_combine, blocks_for(N * R, 256), 256, 0, N, R, j, vstride, Zv, ybuf, kcap, x);
    } else {
      DMB_LAUNCH(c, k_combine, blocks_for(N * R, 256), 256, 0, N, R, j, vstride, V, ybuf, kcap, x);
    }
    DMB_CUDA(cudaMemcpyAsync(hst.data(), st, sizeof(SysState) * R, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
    {
      int kmax = 0;
      for (auto &s : hst) kmax = std::max(kmax, s.k);
      iters_used += kmax;
    }
    bool all_done = true;
    for (auto &s : hst)
      if (!s.done) all_done = false;
    if (all_done && !inexact) break;
    if (!all_done && total_iters >= maxiter) break;
  }
  unsigned e = read_err_word(c);
  DMB_REQUIRE((e & 4u) == 0, DMB_ERR_TIMEOUT, "triangular solve wait expired");
  if (inexact) DMB_REQUIRE(tc_error_word(c) == 0, DMB_ERR_TIMEOUT, "tensor-core GEMM: a pipeline wait expired");
  if (R >= 32 && oz_available(c))
    DMB_REQUIRE(oz_error_word(c) == 0, DMB_ERR_TIMEOUT, "int8 tensor-core GEMM: a pipeline wait expired");
  // true FP64 residual ||b - Z x|| / ||b|| per system
  if (!have_true) {
    if (prod_resid && cycles == 1) {
      // x = sum y_i z_i from x = 0: b - sum y_i (Z z_i) with the stored products
      DMB_LAUNCH(c, k_resid_products, blocks_for(N * R, 256), 256, 0, N, R, j_last, vstride, Wraw, ybuf, kcap, b,
                 w);
    } else {
      matvec_dev(c, x, w, R);
      DMB_LAUNCH(c, k_sub, blocks_for(N * R, 256), 256, 0, N * R, b, w);
    }
    DMB_LAUNCH(c, k_norms, (unsigned)R, 256, 0, N, w, tnrm);
  }
  DMB_LAUNCH(c, k_norms, (unsigned)R, 256, 0, N, b, nrm + R);
  DMB_CUDA(cudaMemcpyAsync(hn_final.data(), nrm + R, 16 * R, cudaMemcpyDeviceToHost, c->stream));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  // The true-residual check: a system that stopped on its recurrence estimate (or on the
  // preconditioned residual, for left preconditioning) with a true residual
  // above tol is refined by another cycle from its current x; that cycle must
  // reduce its starting residual by the factor the true residual still needs
  // (with a margin of 2).
  if (!c->true_residual_check || total_iters >= maxiter || check_pass >= 16) break;
  bool refine = false;
  for (int64_t r = 0; r < R; r++) {
    const double bn = hn_final[r], rn = hn_final[R + r];
    if (!(bn > 0) || !std::isfinite(rn) || rn <= tol * bn || hst[r].done == 3) continue;
    hst[r].done = 0;
    recheck_scale[r] = std::min(0.5, 0.5 * tol * bn / rn);
    refine = true;
  }
  if (!refine) break;
  have_true = false;
  }  // check passes
  const std::vector<double> &hn = hn_final;
  double tres = 0, eres = 0;
  bool solved = true;
  for (int64_t r = 0; r < R; r++) {
    const double bn = hn[r], rn = hn[R + r];
    double rel = bn > 0 ? rn / bn : (rn > 0 ? INFINITY : 0.0);
    tres = std::max(tres, rel);
    double est = hst[r].beta > 0 ? hst[r].resid / hst[r].beta : 0.0;
    if (hst[r].done == 1 || hst[r].done == 2) {
      if (hst[r].done == 1) eres = std::max(eres, est);
    } else {
      solved = false;
      eres = std::max(eres, est);
    }
    if (!std::isfinite(rel)) solved = false;
    if (c->true_residual_check && !(rel <= tol)) solved = false;
  }
  out->niter = iters_used;
  out->solved = solved ? 1 : 0;
  out->residual = eres;
  out->true_residual = tres;
  out->restarts = restarts;
  out->reserved = recheck_continuations;
  c->tm.solve_ms = now_ms() - t0;
  c->tm.gmres_ms = c->tm.solve_ms;
}

}  // namespace dmb
