// dmb_internal.h -- shared declarations of libdiffmom_b200 (not installed).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <array>
#include <chrono>
#include <mutex>
#include <string>
#include <atomic>
#include <map>
#include <vector>

#include "../../include/diffmom_b200.h"

// ---------------------------------------------------------------------------
// error plumbing
// ---------------------------------------------------------------------------
struct DmbError {
  int code;
  std::string msg;
};

#define DMB_CUDA(call)                                                              \
  do {                                                                              \
    cudaError_t e__ = (call);                                                       \
    if (e__ != cudaSuccess)                                                         \
      throw DmbError{DMB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e__)}; \
  } while (0)

#define DMB_REQUIRE(cond, code, text)                 \
  do {                                                \
    if (!(cond)) throw DmbError{(code), (text)};      \
  } while (0)

// message of the calling thread's last failed entry point that takes no
// context (returned by dmb_last_error(NULL))
inline std::string &dmb_free_error() {
  thread_local std::string msg = "null context";
  return msg;
}

// ---------------------------------------------------------------------------
// device buffer (grow-only, owned by the context)
// ---------------------------------------------------------------------------
// bumped by every device (re)allocation or release of a DevBuf: captured CUDA
// graphs hold raw device addresses and are valid only for the epoch they were
// captured in
inline std::atomic<uint64_t> g_dev_alloc_epoch{0};

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  template <class T> T *as() const { return static_cast<T *>(p); }
  void ensure(size_t want) {
    if (want <= bytes && p) return;
    release();
    if (want == 0) want = 16;
    g_dev_alloc_epoch++;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
      p = nullptr;
      bytes = 0;
      throw DmbError{DMB_ERR_BUDGET, std::string("device allocation of ") + std::to_string(want) +
                                         " bytes failed: " + cudaGetErrorString(e)};
    }
    bytes = want;
  }
  void release() {
    if (p) {
      g_dev_alloc_epoch++;
      cudaFree(p);
    }
    p = nullptr;
    bytes = 0;
  }
};

// ---------------------------------------------------------------------------
// per-triangle cache (device, FP64).  Quadrature points are stored both in
// global coordinates (FP64 path, as the reference's cache) and relative to the
// triangle centroid (used by the moment contractions and the FP32 far pairs).
// ---------------------------------------------------------------------------
struct TriCache {
  double v[3][3];     // vertices
  double cen[3];      // centroid
  double area;        // triangle_area
  double w2a[7];      // w_q * 2A for the standard rule
  double w2ah[7];     // w_q * 2A for the 7-point rule
  double qp[7][3];    // standard-rule points (global)
  double qph[7][3];   // 7-point-rule points (global)
  double ql[7][3];    // standard-rule points minus centroid
  // basis slots: RWG functions supported on this triangle (<= 3)
  int rwg[3];         // RWG index (0-based) or -1
  int side[3];        // 0 = T+, 1 = T-
  double s[3];        // signed scale: f(r) = s * (r - p)
  double dv[3];       // surface divergence (+len/A+ or -len/A-)
  double p[3][3];     // opposite vertex (global)
  double pl[3][3];    // opposite vertex minus centroid
};

// near-field record: one (near triangle pair, test slot, source slot)
struct NearRec {
  int ta, tb;     // ta == tb: self; otherwise ta outer (test), tb analytic (source)
  int ia, ib;     // slots
};

// H-matrix operator of dmb_aca_build (dmb_aca.cu).  Blocks are kept in task
// order; their data lives in one complex128 arena (dense: m x n column-major;
// low-rank: U m x rmax then V n x rmax, both column-major).
struct AcaBlockDesc {
  int64_t off_a, off_b;  // arena offsets (complex entries) of data / U and of V
  int32_t r0, m, c0, n;  // tree-order row / column ranges (0-based first, count)
  int32_t kind;          // 0 dense, 1 low-rank
  int32_t rmax;          // capacity of U / V columns (low-rank)
  int32_t task;          // index in the task list
  int32_t fallback;      // 1: admissible task stored dense
};
struct AcaState {
  bool valid = false;
  int64_t n = 0;
  std::vector<int32_t> perm;        // tree order -> original index (0-based)
  std::vector<AcaBlockDesc> blocks; // task order
  std::vector<int32_t> rank;        // per block (low-rank), from the device
  dmb_aca_info info{};
  // device: permutation, blocks, arena, per-block ranks / status, product lists
  DevBuf d_perm, d_blocks, d_arena, d_rank, d_tbuf_off, d_t, d_xp;
  DevBuf d_lr_list;                       // low-rank block ids (inner-product kernel)
  DevBuf d_row_off, d_col_off;            // per row / column leaf: its items (covering blocks, dense first)
  DevBuf d_leaf;                          // leaf node ranges (first, count)
  DevBuf d_zoff_r, d_zoff_c, d_z;         // per-block partial products (row / column side)
  DevBuf d_row_zbase, d_col_zbase;        // per leaf item: partial offset minus the block's first row / column
  int64_t n_leaves = 0, n_lr = 0, t_total = 0;
  double k = 0, eta0 = 0;
  int quad_order = 3;
  void release() {
    DevBuf *b[] = {&d_perm, &d_blocks, &d_arena, &d_rank, &d_tbuf_off, &d_t, &d_xp, &d_lr_list,
                   &d_row_off, &d_col_off, &d_leaf, &d_zoff_r, &d_zoff_c, &d_z,
                   &d_row_zbase, &d_col_zbase};
    for (DevBuf *x : b) x->release();
    valid = false;
  }
};

namespace dmb {
// families of the online autotuner (dmb_tune.cu)
enum TuneFamily { TUNE_TC_GEMM_BN = 0, TUNE_TC_SYRK_STAGES = 1, TUNE_OZ_TILE = 2, TUNE_FAMILIES = 3 };
struct TuneMark {
  bool active = false;
  int family = 0, cand = 0;
  int64_t b1 = 0, b2 = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
};
}  // namespace dmb

// Panels of the far-pair tile kernel (dmb_fartile.cu) for one precision:
// per RWG tile of width T the triangles carrying its functions, packed from
// the per-triangle cache; valid for one (T, quadrature size, cache build).
struct FarTileState {
  bool valid = false;
  int T = 0, nq = 0, ntiles = 0;
  uint64_t cache_gen = 0;
  int64_t ntasks = 0;
  DevBuf d_panels, d_cnt, d_tasks, d_job, d_err;
};

struct dmb_ctx {
  int device = 0;
  // operator of dmb_gmres / dmb_matvec: 0 the resident dense Z, 1 the
  // H-matrix of dmb_aca_build; aca_transposed: products use A^T (the adjoint
  // GMRES solves conj-transformed systems)
  int op_kind = 0;
  bool aca_transposed = false;
  AcaState aca;
  cudaStream_t stream = nullptr;
  // factorisation lookahead (created on first use): stream2 takes the rest of
  // each block column's updates, stream3 the trailing matrix beyond the next
  // block column
  cudaStream_t stream2 = nullptr, stream3 = nullptr;
  cudaEvent_t la_ev[4] = {nullptr, nullptr, nullptr, nullptr};
  // work that only needs Z (right-hand sides, int8 slices of Z) runs here
  // beside the factorisation (created on first use, low priority)
  cudaStream_t stream_aux = nullptr;
  cudaEvent_t aux_ev[2] = {nullptr, nullptr};
  std::mutex mu;
  std::string err;
  int sm_count = 148;

  // mesh / basis (host copies, 0-based)
  int64_t nv = 0, nt = 0, n = 0;
  std::vector<double> h_xyz;
  std::vector<int32_t> h_tri;
  std::vector<int32_t> h_tplus, h_tminus, h_vpo, h_vmo;
  std::vector<double> h_len, h_ap, h_am;
  bool have_mesh = false, have_rwg = false, cache_valid = false;
  int cache_quad_order = 0;
  uint64_t cache_gen = 0;  // bumped by every rebuild of the per-triangle cache

  // device geometry
  DevBuf d_xyz, d_tri, d_tcache, d_rwg_slot;  // rwg_slot: 2 ints per RWG (3t+i)
  DevBuf d_tplus, d_tminus;                   // int32
  DevBuf d_vpo, d_vmo;                        // int32 opposite vertices (0-based)
  DevBuf d_len, d_ap, d_am;                   // RWG edge length / areas
  DevBuf d_slot_rwg, d_slot_side;             // 3 per triangle
  DevBuf d_wq;                                // 7 standard + 7 high-order weights
  DevBuf d_centers;                           // RWG centres (N x 3)
  int nq = 3;
  double wq[7], wqh[7];
  double xi1[7], xi2[7], xh1[7], xh2[7];

  // adjacency + near records
  std::vector<int32_t> adj_off, adj_nb;
  DevBuf d_adj_off, d_adj_nb;
  DevBuf d_near_rec, d_near_val, d_near_entry_mn, d_near_entry_off;
  // the near entries touching each RWG row (CSR, entry order) and the summed
  // value of each entry: the matrix-free product gathers its near part per
  // row in a fixed order (no atomics)
  DevBuf d_near_row_off, d_near_row_ent, d_near_row_col, d_near_entry_sum;
  int64_t n_near_rec = 0, n_near_entry = 0;

  // impedance matrix (row-major == column-major since Z is symmetric)
  DevBuf d_Z;
  int z_prec = -1;    // DMB_PREC_*
  bool z_valid = false;
  double k = 0, eta0 = 376.730313668;
  FarTileState ft[2];  // far-pair tile panels: [0] FP32, [1] FP64

  // preconditioner
  int pc_kind = DMB_PRECOND_NONE;
  int pc_prec = -1;
  DevBuf d_F;         // factor storage (N x N, L strictly lower + D diagonal)
  DevBuf d_dinv;      // Jacobi inverse diagonal
  DevBuf d_W;         // LDL^T panel workspace
  DevBuf d_flags;     // triangular-solve progress flags / error word
  double nnz_ratio = 0;
  bool pc_valid = false;

  // local-inverse / learned preconditioner
  DevBuf d_li_idx, d_li_cnt, d_li_inv;  // neighbour lists and inverse rows
  int li_kmax = 0;
  DevBuf d_net;       // learned weights
  bool net_loaded = false;

  // GMRES workspace (d_Zv: preconditioned basis of the right-preconditioned form)
  DevBuf d_V, d_H, d_work, d_vecs, d_scal, d_Zv;

  // resident solution of dmb_solve_resident / dmb_solve_resident_many
  DevBuf d_rhs, d_sol, d_mono;
  int64_t sol_r = 0;
  // small persistent scratch (counters, plane-wave parameters): the solve path
  // allocates nothing after its first call
  DevBuf d_small;
  bool use_tensor_cores = true;  // complex64 factor update on tcgen05 (else FP32 SIMT)
  int tc_min_rhs = 64;           // batched Z X / triangular solves on tcgen05 from this many RHS
  int far_tile = 0;              // far-pair RWG tile width (FP64 16/32, FP32 32/64), 0 = autotuned
  bool exact_krylov = true;      // many-RHS Krylov product on the INT8 slices (FP64-accurate)
  // GMRES iterations between host checks replayed as captured CUDA graphs
  // (few right-hand sides); key: iteration range, shape, buffer addresses and
  // the allocation epoch
  bool gmres_graphs = true;
  // GMRES tests convergence on ||b - Z x|| / ||b|| (FP64-accurate product):
  // a system whose recurrence estimate met the tolerance but whose true
  // residual did not is refined by further cycles from its current iterate
  bool true_residual_check = true;
  // polls of a triangular-solve chain wait before it gives up (DMB_ERR_TIMEOUT);
  // DMB_OPT_SPIN_LIMIT lowers it to exercise the timeout path
  long long spin_limit = 20000000;
  struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    int64_t kernels = 0;
    bool seen = false;
  };
  std::map<std::vector<int64_t>, GraphEntry> gm_graphs;
  int precond_tf32_terms = 3;    // TF32 products of the complex64 factor updates and packed sweeps (3 or 1)
  // those operands split into BF16 pieces (kind::f16 MMA) instead of TF32:
  // 1 always, 0 never, -1 (default) inside the resident solves only
  // (dmb_solve_resident[_many], batch surfaces: pc_bf16_scope set), whose
  // GMRES is checked on the FP64 residual, so the preconditioner's precision is
  // a matter of iteration count alone
  int precond_bf16 = -1;
  int int8_scheme = 0;  // FP64-accurate INT8 product: 0 residues modulo coprime moduli (CRT), 1 fixed-point slices
  bool pc_bf16_scope = false;
  bool pc_bf16() const { return precond_bf16 > 0 || (precond_bf16 < 0 && pc_bf16_scope); }
  int far_tile_used = 0;         // tile width of the last assembly
  // autotuner pins per family (0: tuned, k: candidate k - 1)
  int tune_pin[dmb::TUNE_FAMILIES] = {0, 0, 0};
  uint64_t z_version = 0;        // bumped whenever Z changes (packed operand caches key on it)
  uint64_t f_version = 0;        // bumped by every LDL^T factorisation
  uint64_t f_packed = ~0ull;     // factor version packed for the batched triangular solves
  uint64_t f_inv = ~0ull;        // factor version whose 1024-row block inverses are in d_trsm_id
  uint64_t f_inv64 = ~0ull;      // ... whose FP64-product block inverses are in d_sv_inv
  DevBuf d_sv_acc, d_sv_part, d_sv_inv;  // the blocked one-RHS sweeps: scratch and block inverses
  // inputs of the current host topology (build_host_topology)
  bool topo_valid = false;
  std::vector<int32_t> topo_tri, topo_tplus, topo_tminus;
  DevBuf d_trsm_id;              // scratch: inverses of the 1024-row diagonal blocks of L
  DevBuf d_trsm_t;               // scratch: products of the recursive-doubling levels
  int gm_kcap = 0;              // cached GMRES basis capacity
  int64_t gm_key_n = 0, gm_key_r = 0;
  int gm_key_maxiter = 0;
  bool gm_key_flex = false;
  int gm_key_nvec = 0;          // basis-sized vectors kept per iteration
  DevBuf d_Wraw;                // Z z_i before orthogonalisation (residual from the Krylov products)

  // timings
  dmb_timings tm{};
  int64_t launches = 0;
  bool kt_enabled = false;     // dominant-kernel event timing
  // per family: 0 3xTF32 Krylov / sweep GEMMs, 1 int8 GEMMs, 2 factor updates,
  // 3 H-matrix products (one right-hand side, work in bytes), 4 FP64-pipe
  // complex128 Z X and sweep GEMMs, 5 far-pair tiles of the assembly (work in
  // bytes of Z written)
  static constexpr int KT_FAMILIES = 6;
  double kt_ms[KT_FAMILIES] = {0, 0, 0, 0, 0, 0}, kt_flops[KT_FAMILIES] = {0, 0, 0, 0, 0, 0};
  int64_t kt_launches[KT_FAMILIES] = {0, 0, 0, 0, 0, 0};
  std::vector<cudaEvent_t> kt_pool;   // (start, end) pairs recorded around launches
  std::vector<double> kt_pending;     // algorithmic work of each recorded launch
  std::vector<int> kt_family;         // family of each recorded launch
  size_t kt_used = 0;
};

// Bracket one launch of a timed kernel family with events from a pre-created
// pool (no host synchronisation inside the timed region).
inline void kt_begin(dmb_ctx *c) {
  if (!c->kt_enabled) return;
  if (c->kt_used + 2 > c->kt_pool.size()) {
    for (int i = 0; i < 256; i++) {
      cudaEvent_t e;
      DMB_CUDA(cudaEventCreate(&e));
      c->kt_pool.push_back(e);
    }
  }
  DMB_CUDA(cudaEventRecord(c->kt_pool[c->kt_used], c->stream));
}
inline void kt_end(dmb_ctx *c, double work, int family = 0) {
  if (!c->kt_enabled) return;
  DMB_CUDA(cudaEventRecord(c->kt_pool[c->kt_used + 1], c->stream));
  c->kt_used += 2;
  c->kt_pending.push_back(work);
  c->kt_family.push_back(family);
}
// fold the recorded pairs into the totals (synchronises the device work)
inline void kt_collect(dmb_ctx *c) {
  if (c->kt_used == 0) return;
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  for (size_t i = 0; i + 1 < c->kt_used; i += 2) {
    float ms = 0;
    DMB_CUDA(cudaEventSynchronize(c->kt_pool[i + 1]));
    DMB_CUDA(cudaEventElapsedTime(&ms, c->kt_pool[i], c->kt_pool[i + 1]));
    const int f = c->kt_family[i / 2];
    c->kt_ms[f] += ms;
    c->kt_launches[f]++;
    c->kt_flops[f] += c->kt_pending[i / 2];
  }
  c->kt_used = 0;
  c->kt_pending.clear();
  c->kt_family.clear();
}

// Runs the enclosed launches of a context on another stream (the context is
// used by one thread at a time).
struct StreamSwap {
  dmb_ctx *c;
  cudaStream_t saved;
  StreamSwap(dmb_ctx *ctx, cudaStream_t s) : c(ctx), saved(ctx->stream) { ctx->stream = s; }
  ~StreamSwap() { c->stream = saved; }
};

// ---------------------------------------------------------------------------
// helpers shared by translation units
// ---------------------------------------------------------------------------
namespace dmb {
void ensure_cache(dmb_ctx *c, int quad_order);
void gradient_impedance_dev(dmb_ctx *c, int64_t R, const double2 *I_dev, const double2 *L_dev,
                            const int *tri_patch, int64_t P, int reactive, int quad_order, double *g_dev);
void build_host_topology(dmb_ctx *c);
// far-pair part of Z by RWG tiles (dmb_fartile.cu)
bool far_tile_width_valid(int T, bool f64);
void far_panels(dmb_ctx *c, int T, bool f64);
void far_tiles(dmb_ctx *c, int T, bool f64, double k, double inv_k2, double omega_mu0);
int far_tile_width(dmb_ctx *c, bool f64, double k, double inv_k2, double omega_mu0);
int far_tile_width_known(dmb_ctx *c, int64_t n, bool f64);  // 0: not tuned yet
unsigned far_error_word(dmb_ctx *c, bool f64);
void far_release(dmb_ctx *c);
void far_tiles_batched(const std::vector<dmb_ctx *> &cs, int T, bool f64, double k, double inv_k2,
                       double omega_mu0, DevBuf &d_jobs, DevBuf &d_tasks, DevBuf &d_err);
// impedance matrices of many surfaces: far tiles in one launch, near values
// and near sums in one launch each, on the stream of cs[0] (dmb_assemble.cu);
// returns the device time of the three launches
struct BatchAsmBufs {
  DevBuf far_jobs, far_tasks, far_err, near_jobs;
};
double assemble_batch(const std::vector<dmb_ctx *> &cs, double k, double eta0, int quad_order, int precision,
                      BatchAsmBufs &bufs);
// online autotuner (dmb_tune.cu): candidate for a (family, bucket), and the
// event bracket of a launch while the bucket is being measured
int64_t tune_bucket(int64_t v);  // floor(log2(v))
int tune_choose(dmb_ctx *c, int family, int64_t b1, int64_t b2, int ncand);
bool tune_begin(dmb_ctx *c, int family, int64_t b1, int64_t b2, int cand, TuneMark &mk);
void tune_end(dmb_ctx *c, TuneMark &mk);
std::string tune_report();
void assemble(dmb_ctx *c, double k, double eta0, int quad_order, int precision);
void copy_z_out(dmb_ctx *c, double *Z_out);
void z_entries(dmb_ctx *c, const int64_t *m, const int64_t *n, int64_t count, double *out);
void apply_impedance(dmb_ctx *c, const double *zs);
// FP64 complex GEMMs on the FP64 pipe (dmb_zgemm64.cu): Y = Z X (column-major
// N x R), Y(m, r) -= sum_k A(m, k) B[r ldb + k] (A(m, k) = A[m lda + k], or
// A[k lda + m] when a_transposed; Y column-major), and the lower-triangle
// trailing update F[m][j] -= sum_k W[m][k] L[j][k] (row-major, j <= m)
void zgemm64_zx(dmb_ctx *c, const double2 *Z, const double2 *X, double2 *Y, int64_t N, int64_t R);
void zgemm64_sub(dmb_ctx *c, bool a_transposed, int64_t M, int64_t R, int64_t K, const double2 *A, int64_t lda,
                 const double2 *B, int64_t ldb, double2 *Y, int64_t ldy);
void zgemm64_lower_update(dmb_ctx *c, int64_t M, int64_t C, int64_t K, const double2 *W, int64_t ldw,
                          const double2 *Lrows, int64_t ldl, double2 *F, int64_t ldf);
unsigned read_err_word(dmb_ctx *c);  // error word of the triangular solves (bit 2: a wait expired)
void matvec_dev(dmb_ctx *c, const void *x, void *y, int64_t nrhs);  // device buffers, c128
void conj_dev(dmb_ctx *c, double2 *x, int64_t count);
void nf_build(dmb_ctx *c, double cutoff, int kind);
void pc_apply_dev(dmb_ctx *c, double *x, int64_t nrhs);             // in place, c128 device
void rhs_plane_waves_dev(dmb_ctx *c, const double *kvecs, const double *E0s, const double *pols,
                         int64_t R, int quad_order, double *V_dev);
void rhs_plane_waves_async(dmb_ctx *c, const double *kvecs, const double *E0s, const double *pols, int64_t R,
                           int quad_order, double *V_dev);
void rhs_dipoles_dev(dmb_ctx *c, int64_t R, const double *pos, const double *moments, const int *magnetic,
                     const double *freqs, int quad_order, double *V_dev);
void rhs_pattern_dev(dmb_ctx *c, int nth, const double *theta, int nph, const double *phi, const double *Ft,
                     const double *Fp, double freq, const double *pc, int conj_conv, int quad_order, double *V_dev);
void gmres_dev(dmb_ctx *c, const double *b_dev, double *x_dev, int64_t nrhs, double tol,
               int maxiter, int precond_kind, int precond_side, dmb_gmres_stats *st);
void solve_direct_dev(dmb_ctx *c, const double *b_dev, double *x_dev, int64_t nrhs,
                      double *berr);
void farfield_dev(dmb_ctx *c, const double *rhat, int64_t NO, double k, double eta0,
                  int quad_order, const double *I_dev, int64_t nrhs, double *E_dev);
void prepare_operator(dmb_ctx *c, double k, double eta0, int quad_order);
void monostatic_dev(dmb_ctx *c, int64_t R, double k, double eta0, int quad_order, const double *I_dev,
                    double *E_dev, double *sigma_dev);
void matvec_free_dev(dmb_ctx *c, const double *x, double *y);
void local_inverse_build(dmb_ctx *c, double radius, int kmax);
// tensor-core complex GEMMs (dmb_tc.cu)
bool tc_available(dmb_ctx *c);
void tc_zx(dmb_ctx *c, const double2 *X, double2 *Y, int64_t R);
void tc_trsm_update(dmb_ctx *c, const float2 *F, int64_t N, int64_t r_lo, int64_t r_hi, int64_t k_lo, int width,
                    bool backward, double2 *X, int64_t R);
void tc_trsm_pack_factor(dmb_ctx *c, const float2 *F, int64_t N);
void tc_trsm_pack_diag(dmb_ctx *c, int64_t o, const double2 *Xb, int64_t ld, int ow);
void tc_trsm_sweep(dmb_ctx *c, int64_t N, double2 *X, int64_t R, bool backward);
unsigned tc_error_word(dmb_ctx *c);
void tc_release(dmb_ctx *c);
// FP64-accurate complex64 Z X on the INT8 tensor cores (dmb_ozaki.cu)
bool oz_available(dmb_ctx *c);
bool krylov_exact_int8(dmb_ctx *c, int64_t nrhs);  // the Krylov product is the INT8-slice one
// lmax: the accuracy class.  Residue scheme: 6 -> 13 moduli (13 int8
// products, ~1e-13 normwise), 5 -> 12 moduli (12 products, ~1e-12).  Slice
// scheme: slice-pair levels p + q <= lmax are kept (6: 26 int8 products,
// ~7e-13; 5: 21 products, ~4e-11 -- enough for the Krylov recurrence)
constexpr int OZ_LEVELS_RESIDUAL = 6, OZ_LEVELS_KRYLOV = 5;
void oz_zx(dmb_ctx *c, const double2 *X, double2 *Y, int64_t R, int lmax = OZ_LEVELS_RESIDUAL);
void oz_prepare(dmb_ctx *c);
unsigned oz_error_word(dmb_ctx *c);
void oz_release(dmb_ctx *c);
void local_release(dmb_ctx *c);
// Krylov operator (may be on the tensor cores); full_levels: the INT8-slice
// product with every slice level (FP64-accurate) instead of the Krylov levels
void matvec_op(dmb_ctx *c, const double2 *x, double2 *y, int64_t nrhs, bool full_levels = false);
bool matvec_op_inexact(dmb_ctx *c, int64_t nrhs);
void learned_build(dmb_ctx *c, double radius);
void ring_step_build(dmb_ctx *c, double radius, bool learned);
void ls_build(dmb_ctx *c, double radius);
void local_apply_dev(dmb_ctx *c, double *x, int64_t nrhs);
double learned_train_body(dmb_ctx *c, double radius, int epochs, int batch, double lr, uint64_t seed);
void net_loss_grad(dmb_ctx *c, const float *feat, const float *tgt, const float *wgt, const int *cnt,
                   int64_t nrows, float *grad, float *loss);
int net_param_count();
void net_set(dmb_ctx *c, const float *w);
void net_get(dmb_ctx *c, float *w);
double now_ms();
// H-matrix operator (dmb_aca.cu): mode 0 A x, 1 A^H x, 2 A^T x on device
// complex128 vectors (nrhs columns)
void aca_apply(dmb_ctx *c, const double2 *x, double2 *y, int64_t nrhs, int mode);
bool operator_ready(dmb_ctx *c);
}  // namespace dmb

// launch bookkeeping: every library kernel launch goes through this macro so
// the context can report how many of its kernels ran.
#define DMB_LAUNCH(ctx, kernel, grid, block, smem, ...)                        \
  do {                                                                         \
    kernel<<<(grid), (block), (smem), (ctx)->stream>>>(__VA_ARGS__);          \
    DMB_CUDA(cudaGetLastError());                                              \
    (ctx)->launches++;                                                         \
  } while (0)
