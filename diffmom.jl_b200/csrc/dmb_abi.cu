// dmb_abi.cu -- extern "C" entry points of libdiffmom_b200.
//
// Each entry point validates its arguments with the reference's fail-closed
// rules, takes the context mutex, runs the device path and maps exceptions to
// status codes.  Host buffers are copied on the context's stream.
#include <cmath>
#include <cstring>

#include <algorithm>
#include <atomic>
#include <thread>
#include <functional>

#include "dmb_device.cuh"
#include "dmb_internal.h"

namespace {

// Marks a resident solve: inside it the complex64 preconditioner's
// tensor-core work may use BF16 operand pieces (DMB_OPT_PRECOND_BF16 = -1).
struct PcBf16Scope {
  dmb_ctx *c;
  explicit PcBf16Scope(dmb_ctx *ctx) : c(ctx) { c->pc_bf16_scope = true; }
  ~PcBf16Scope() { c->pc_bf16_scope = false; }
};

template <class F> dmb_status guarded(dmb_ctx *c, F &&f) {
  if (!c) return DMB_ERR_ARGUMENT;
  std::lock_guard<std::mutex> lk(c->mu);
  try {
    cudaSetDevice(c->device);
    f();
    c->err.clear();
    return DMB_OK;
  } catch (const DmbError &e) {
    c->err = e.msg;
    return e.code;
  } catch (const std::exception &e) {
    c->err = e.what();
    return DMB_ERR_STATE;
  }
}

void check_finite(const double *p, int64_t n, const char *what) {
  for (int64_t i = 0; i < n; i++)
    if (!std::isfinite(p[i]))
      throw DmbError{DMB_ERR_ARGUMENT, std::string(what) + " must contain only finite values"};
}

}  // namespace

extern "C" {

const char *dmb_version(void) { return "diffmom_b200 0.1 sm_100a"; }

dmb_status dmb_ctx_create(int device, dmb_ctx **out) {
  if (!out) return DMB_ERR_ARGUMENT;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return DMB_ERR_CUDA;
  if (device < 0 || device >= count) return DMB_ERR_ARGUMENT;
  dmb_ctx *c = new dmb_ctx();
  c->device = device;
  // the context stream runs at the highest priority: during the factorisation
  // its latency-bound panel chain is scheduled ahead of the lookahead updates
  // queued on the low-priority second stream
  int prio_least = 0, prio_greatest = 0;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest) != cudaSuccess ||
      cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, prio_greatest) != cudaSuccess) {
    delete c;
    return DMB_ERR_CUDA;
  }
  cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
  *out = c;
  return DMB_OK;
}

dmb_status dmb_ctx_destroy(dmb_ctx *c) {
  if (!c) return DMB_OK;
  {
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    DevBuf *bufs[] = {&c->d_xyz, &c->d_tri, &c->d_tcache, &c->d_rwg_slot, &c->d_tplus,
                      &c->d_tminus, &c->d_vpo, &c->d_vmo, &c->d_len, &c->d_ap, &c->d_am,
                      &c->d_slot_rwg, &c->d_slot_side, &c->d_wq, &c->d_centers, &c->d_adj_off,
                      &c->d_adj_nb, &c->d_near_rec, &c->d_near_val, &c->d_near_entry_mn,
                      &c->d_near_entry_off, &c->d_near_row_off, &c->d_near_row_ent, &c->d_near_row_col,
                      &c->d_near_entry_sum, &c->d_Z, &c->d_F, &c->d_dinv, &c->d_W,
                      &c->d_flags, &c->d_li_idx, &c->d_li_cnt, &c->d_li_inv, &c->d_net, &c->d_V,
                      &c->d_H, &c->d_work, &c->d_vecs, &c->d_scal};
    for (DevBuf *b : bufs) b->release();
    c->d_rhs.release();
    c->d_sol.release();
    c->d_mono.release();
    c->d_trsm_id.release();
    c->d_Wraw.release();
    c->d_trsm_t.release();
    c->d_sv_acc.release();
    c->d_sv_part.release();
    c->d_sv_inv.release();
    c->d_Zv.release();
    c->d_small.release();
    c->aca.release();
    dmb::tc_release(c);
    dmb::oz_release(c);
    dmb::local_release(c);
    dmb::far_release(c);
    for (auto &e : c->kt_pool) cudaEventDestroy(e);
    if (c->stream2) cudaStreamDestroy(c->stream2);
    for (auto &kv : c->gm_graphs)
      if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    c->gm_graphs.clear();
    if (c->stream3) cudaStreamDestroy(c->stream3);
    if (c->stream_aux) cudaStreamDestroy(c->stream_aux);
    for (auto &e : c->aux_ev)
      if (e) cudaEventDestroy(e);
    for (auto &e : c->la_ev)
      if (e) cudaEventDestroy(e);
    cudaStreamDestroy(c->stream);
  }
  delete c;
  return DMB_OK;
}

const char *dmb_last_error(const dmb_ctx *c) { return c ? c->err.c_str() : dmb_free_error().c_str(); }

dmb_status dmb_get_timings(dmb_ctx *c, dmb_timings *out) {
  return guarded(c, [&] {
    DMB_REQUIRE(out, DMB_ERR_ARGUMENT, "timings output is NULL");
    c->tm.kernels = c->launches;
    *out = c->tm;
  });
}

dmb_status dmb_set_option(dmb_ctx *c, int option, int value) {
  return guarded(c, [&] {
    if (option == DMB_OPT_TENSOR_CORES) {
      c->use_tensor_cores = value != 0;
      c->pc_valid = false;
      return;
    }
    if (option == DMB_OPT_INT8_SCHEME) {
      DMB_REQUIRE(value == 0 || value == 1, DMB_ERR_ARGUMENT, "int8 scheme must be 0 (residues) or 1 (slices)");
      c->int8_scheme = value;
      return;
    }
    if (option == DMB_OPT_EXACT_KRYLOV) {
      c->exact_krylov = value != 0;
      return;
    }
    if (option == DMB_OPT_FAR_TILE) {
      DMB_REQUIRE(value == 0 || value == 16 || value == 32 || value == 64, DMB_ERR_ARGUMENT,
                  "far tile width must be 0 (autotune), 16, 32 or 64");
      c->far_tile = value;
      return;
    }
    if (option == DMB_OPT_GMRES_GRAPHS) {
      c->gmres_graphs = value != 0;
      return;
    }
    if (option == DMB_OPT_TRUE_RESIDUAL) {
      c->true_residual_check = value != 0;
      return;
    }
    if (option == DMB_OPT_SPIN_LIMIT) {
      c->spin_limit = value < 0 ? 20000000LL : (long long)value;
      return;
    }
    if (option == DMB_OPT_PRECOND_BF16) {
      DMB_REQUIRE(value >= -1 && value <= 1, DMB_ERR_ARGUMENT, "DMB_OPT_PRECOND_BF16 must be -1, 0 or 1");
      if (c->precond_bf16 != value) c->pc_valid = false;
      c->precond_bf16 = value;
      return;
    }
    if (option == DMB_OPT_TUNE_TC_GEMM || option == DMB_OPT_TUNE_TC_SYRK) {
      const int ncand = 3;
      DMB_REQUIRE(value >= 0 && value <= ncand, DMB_ERR_ARGUMENT,
                  "autotuner pin must be 0 (tuned) or a candidate 1.." + std::to_string(ncand));
      c->tune_pin[option == DMB_OPT_TUNE_TC_GEMM ? dmb::TUNE_TC_GEMM_BN : dmb::TUNE_TC_SYRK_STAGES] = value;
      return;
    }
    if (option == DMB_OPT_TUNE_INT8_TILE) {
      DMB_REQUIRE(value >= 0 && value <= 2, DMB_ERR_ARGUMENT, "int8 tile pin must be 0 (tuned), 1 or 2");
      c->tune_pin[dmb::TUNE_OZ_TILE] = value;
      return;
    }
    if (option == DMB_OPT_OPERATOR) {
      DMB_REQUIRE(value == 0 || value == 1, DMB_ERR_ARGUMENT, "operator must be 0 (dense Z) or 1 (H-matrix)");
      DMB_REQUIRE(value == 0 ? c->z_valid : c->aca.valid, DMB_ERR_STATE,
                  value == 0 ? "no assembled impedance matrix" : "no H-matrix operator built");
      if (c->op_kind != value) c->pc_valid = false;
      c->op_kind = value;
      return;
    }
    if (option == DMB_OPT_PRECOND_TF32_TERMS) {
      DMB_REQUIRE(value == 1 || value == 3, DMB_ERR_ARGUMENT, "TF32 products per complex64 factor MAC must be 1 or 3");
      c->precond_tf32_terms = value;
      c->pc_valid = false;
      return;
    }
    if (option == DMB_OPT_TC_MIN_RHS) {
      DMB_REQUIRE(value >= 1, DMB_ERR_ARGUMENT, "minimum right-hand-side count must be >= 1");
      c->tc_min_rhs = value;
      return;
    }
    throw DmbError{DMB_ERR_ARGUMENT, "unknown option " + std::to_string(option)};
  });
}

dmb_status dmb_get_far_tile(dmb_ctx *c, int *width_out) {
  return guarded(c, [&] {
    DMB_REQUIRE(width_out, DMB_ERR_ARGUMENT, "output is NULL");
    *width_out = c->far_tile_used;
  });
}

dmb_status dmb_tune_report(char *buf, size_t cap, size_t *len_out) {
  try {
    const std::string r = dmb::tune_report();
    if (len_out) *len_out = r.size();
    if (buf && cap > 0) {
      const size_t n = std::min(cap - 1, r.size());
      std::memcpy(buf, r.data(), n);
      buf[n] = 0;
    }
    return DMB_OK;
  } catch (const DmbError &e) {
    dmb_free_error() = e.msg;
    return (dmb_status)e.code;
  }
}

dmb_status dmb_mesh_upload(dmb_ctx *c, const double *xyz, const int64_t *tri, int64_t nv, int64_t nt) {
  return guarded(c, [&] {
    DMB_REQUIRE(xyz && tri, DMB_ERR_ARGUMENT, "mesh arrays must be non-NULL");
    DMB_REQUIRE(nv >= 3 && nt >= 1, DMB_ERR_ARGUMENT, "mesh needs at least 3 vertices and 1 triangle");
    DMB_REQUIRE(nt < (1LL << 28) && nv < (1LL << 30), DMB_ERR_BUDGET, "mesh exceeds supported size");
    check_finite(xyz, 3 * nv, "mesh coordinates");
    c->h_xyz.assign(xyz, xyz + 3 * nv);
    c->h_tri.resize(3 * nt);
    for (int64_t i = 0; i < 3 * nt; i++) {
      DMB_REQUIRE(tri[i] >= 1 && tri[i] <= nv, DMB_ERR_ARGUMENT,
                  "triangle vertex index out of range at position " + std::to_string(i + 1));
      c->h_tri[i] = (int32_t)(tri[i] - 1);
    }
    c->nv = nv;
    c->nt = nt;
    c->d_xyz.ensure(sizeof(double) * 3 * nv);
    c->d_tri.ensure(sizeof(int32_t) * 3 * nt);
    DMB_CUDA(cudaMemcpyAsync(c->d_xyz.p, c->h_xyz.data(), sizeof(double) * 3 * nv, cudaMemcpyHostToDevice, c->stream));
    DMB_CUDA(cudaMemcpyAsync(c->d_tri.p, c->h_tri.data(), sizeof(int32_t) * 3 * nt, cudaMemcpyHostToDevice, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
    c->have_mesh = true;
    c->have_rwg = false;
    c->cache_valid = false;
    c->z_valid = false;
    c->pc_valid = false;
    c->aca.release();
    c->op_kind = 0;
  });
}

dmb_status dmb_rwg_upload(dmb_ctx *c, int64_t n, const int64_t *tplus, const int64_t *tminus,
                          const int64_t *evert, const int64_t *vplus_opp, const int64_t *vminus_opp,
                          const double *len, const double *area_plus, const double *area_minus) {
  return guarded(c, [&] {
    DMB_REQUIRE(c->have_mesh, DMB_ERR_STATE, "upload the mesh before the RWG data");
    DMB_REQUIRE(n >= 1, DMB_ERR_ARGUMENT,
                "mesh produces no RWG unknowns; at least two triangles sharing an edge are required");
    DMB_REQUIRE(tplus && tminus && vplus_opp && vminus_opp && len && area_plus && area_minus,
                DMB_ERR_ARGUMENT, "RWG arrays must be non-NULL");
    DMB_REQUIRE(n <= 3 * c->nt, DMB_ERR_DIMENSION, "more RWG functions than triangle edges");
    auto idx = [&](const int64_t *a, int64_t lim, std::vector<int32_t> &o, const char *what) {
      o.resize(n);
      for (int64_t i = 0; i < n; i++) {
        DMB_REQUIRE(a[i] >= 1 && a[i] <= lim, DMB_ERR_ARGUMENT,
                    std::string(what) + " index out of range at RWG " + std::to_string(i + 1));
        o[i] = (int32_t)(a[i] - 1);
      }
    };
    idx(tplus, c->nt, c->h_tplus, "tplus");
    idx(tminus, c->nt, c->h_tminus, "tminus");
    idx(vplus_opp, c->nv, c->h_vpo, "vplus_opp");
    idx(vminus_opp, c->nv, c->h_vmo, "vminus_opp");
    for (int64_t i = 0; i < n; i++) {
      DMB_REQUIRE(c->h_tplus[i] != c->h_tminus[i], DMB_ERR_ARGUMENT,
                  "RWG " + std::to_string(i + 1) + " has identical T+ and T-");
      DMB_REQUIRE(std::isfinite(len[i]) && len[i] > 0, DMB_ERR_ARGUMENT,
                  "RWG edge has zero or unrepresentable length");
      DMB_REQUIRE(std::isfinite(area_plus[i]) && area_plus[i] > 0 && std::isfinite(area_minus[i]) &&
                      area_minus[i] > 0,
                  DMB_ERR_ARGUMENT, "RWG triangle areas must be finite and positive");
    }
    (void)evert;
    c->h_len.assign(len, len + n);
    c->h_ap.assign(area_plus, area_plus + n);
    c->h_am.assign(area_minus, area_minus + n);
    c->n = n;
    auto up = [&](DevBuf &b, const void *src, size_t bytes) {
      b.ensure(bytes);
      DMB_CUDA(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, c->stream));
    };
    up(c->d_tplus, c->h_tplus.data(), 4 * n);
    up(c->d_tminus, c->h_tminus.data(), 4 * n);
    up(c->d_vpo, c->h_vpo.data(), 4 * n);
    up(c->d_vmo, c->h_vmo.data(), 4 * n);
    up(c->d_len, c->h_len.data(), 8 * n);
    up(c->d_ap, c->h_ap.data(), 8 * n);
    up(c->d_am, c->h_am.data(), 8 * n);
    // the edge adjacency, basis slots and near-field records depend only on
    // the triangles and the RWG triangle pairs: an identical re-upload keeps them
    if (!(c->topo_valid && c->topo_tri == c->h_tri && c->topo_tplus == c->h_tplus &&
          c->topo_tminus == c->h_tminus)) {
      c->topo_valid = false;
      dmb::build_host_topology(c);
      c->topo_tri = c->h_tri;
      c->topo_tplus = c->h_tplus;
      c->topo_tminus = c->h_tminus;
      c->topo_valid = true;
    }
    c->have_rwg = true;
    c->cache_valid = false;
    c->z_valid = false;
    c->pc_valid = false;
    c->aca.release();
    c->op_kind = 0;
  });
}

dmb_status dmb_assemble_z(dmb_ctx *c, double k, double eta0, int quad_order, int precision,
                          double *Z_out) {
  return guarded(c, [&] {
    dmb::assemble(c, k, eta0, quad_order, precision);
    if (Z_out) dmb::copy_z_out(c, Z_out);
  });
}

dmb_status dmb_z_entries(dmb_ctx *c, const int64_t *m, const int64_t *n, int64_t count, double *out) {
  return guarded(c, [&] {
    DMB_REQUIRE(c->z_valid, DMB_ERR_STATE, "no assembled impedance matrix");
    DMB_REQUIRE(count >= 0 && (count == 0 || (m && n && out)), DMB_ERR_ARGUMENT, "bad entry arrays");
    for (int64_t i = 0; i < count; i++)
      DMB_REQUIRE(m[i] >= 1 && m[i] <= c->n && n[i] >= 1 && n[i] <= c->n, DMB_ERR_ARGUMENT,
                  "entry index out of range");
    dmb::z_entries(c, m, n, count, out);
  });
}

dmb_status dmb_apply_impedance(dmb_ctx *c, const double *zs) {
  return guarded(c, [&] {
    DMB_REQUIRE(c->z_valid, DMB_ERR_STATE, "no assembled impedance matrix");
    DMB_REQUIRE(zs, DMB_ERR_ARGUMENT, "surface impedance array is NULL");
    check_finite(zs, 2 * c->nt, "surface impedance");
    dmb::apply_impedance(c, zs);
  });
}

dmb_status dmb_matvec(dmb_ctx *c, const double *x, double *y, int64_t nrhs) {
  return guarded(c, [&] {
    DMB_REQUIRE(dmb::operator_ready(c), DMB_ERR_STATE, "no assembled impedance matrix");
    DMB_REQUIRE(x && y && nrhs >= 1, DMB_ERR_ARGUMENT, "bad matvec arguments");
    size_t bytes = sizeof(double2) * c->n * nrhs;
    DevBuf bx, by;
    bx.ensure(bytes);
    by.ensure(bytes);
    DMB_CUDA(cudaMemcpyAsync(bx.p, x, bytes, cudaMemcpyHostToDevice, c->stream));
    // the 3xTF32 operator when it is the Krylov operator, else the
    // FP64-accurate product (every int8 slice level for many columns)
    if (dmb::matvec_op_inexact(c, nrhs)) {
      dmb::matvec_op(c, bx.as<double2>(), by.as<double2>(), nrhs);
      DMB_REQUIRE(dmb::tc_error_word(c) == 0, DMB_ERR_TIMEOUT, "tensor-core GEMM: a pipeline wait expired");
    } else {
      dmb::matvec_dev(c, bx.as<double2>(), by.as<double2>(), nrhs);
    }
    DMB_CUDA(cudaMemcpyAsync(y, by.p, bytes, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
  });
}

dmb_status dmb_prepare_operator(dmb_ctx *c, double k, double eta0, int quad_order) {
  return guarded(c, [&] { dmb::prepare_operator(c, k, eta0, quad_order); });
}

dmb_status dmb_matvec_free(dmb_ctx *c, const double *x, double *y) {
  return guarded(c, [&] {
    DMB_REQUIRE(x && y, DMB_ERR_ARGUMENT, "bad matvec arguments");
    size_t bytes = sizeof(double2) * c->n;
    DevBuf bx, by;
    bx.ensure(bytes);
    by.ensure(bytes);
    DMB_CUDA(cudaMemcpyAsync(bx.p, x, bytes, cudaMemcpyHostToDevice, c->stream));
    dmb::matvec_free_dev(c, bx.as<double>(), by.as<double>());
    DMB_CUDA(cudaMemcpyAsync(y, by.p, bytes, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
  });
}

dmb_status dmb_nf_build(dmb_ctx *c, double cutoff, int kind, double *nnz_ratio_out) {
  return guarded(c, [&] {
    DMB_REQUIRE(!std::isnan(cutoff) && cutoff >= 0.0, DMB_ERR_ARGUMENT,
                "near-field cutoff must be nonnegative and not NaN");
    DMB_REQUIRE(kind == DMB_PRECOND_NF_LU || kind == DMB_PRECOND_NF_DIAG, DMB_ERR_ARGUMENT,
                "invalid factorization; expected :lu or :diag");
    DMB_REQUIRE(c->z_valid, DMB_ERR_STATE, "no assembled impedance matrix");
    DMB_REQUIRE(c->op_kind == 0, DMB_ERR_STATE,
                "the operator is an H-matrix: build its near-field preconditioner with dmb_aca_nf_build");
    dmb::nf_build(c, cutoff, kind);
    if (nnz_ratio_out) *nnz_ratio_out = c->nnz_ratio;
  });
}

dmb_status dmb_nf_apply(dmb_ctx *c, const double *x, double *y, int64_t nrhs) {
  return guarded(c, [&] {
    DMB_REQUIRE(c->pc_valid, DMB_ERR_STATE, "no near-field preconditioner built");
    DMB_REQUIRE(x && y && nrhs >= 1, DMB_ERR_ARGUMENT, "bad apply arguments");
    size_t bytes = sizeof(double2) * c->n * nrhs;
    DevBuf bx;
    bx.ensure(bytes);
    DMB_CUDA(cudaMemcpyAsync(bx.p, x, bytes, cudaMemcpyHostToDevice, c->stream));
    dmb::pc_apply_dev(c, bx.as<double>(), nrhs);
    DMB_CUDA(cudaMemcpyAsync(y, bx.p, bytes, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
    DMB_REQUIRE((dmb::read_err_word(c) & 4u) == 0, DMB_ERR_TIMEOUT, "triangular solve wait expired");
  });
}

dmb_status dmb_local_build(dmb_ctx *c, double radius, int mode) {
  return guarded(c, [&] {
    DMB_REQUIRE(mode >= 0 && mode <= 3, DMB_ERR_ARGUMENT, "local preconditioner mode must be 0, 1, 2 or 3");
    if (mode == 1)
      dmb::learned_build(c, radius);
    else if (mode == 2)
      dmb::ls_build(c, radius);
    else if (mode == 3)
      dmb::ring_step_build(c, radius, false);
    else
      dmb::local_inverse_build(c, radius, 64);
  });
}

dmb_status dmb_net_train(dmb_ctx *c, double radius, int epochs, int batch, double lr, uint64_t seed,
                         double *loss_out) {
  return guarded(c, [&] {
    DMB_REQUIRE(std::isfinite(lr) && lr > 0, DMB_ERR_ARGUMENT, "learning rate must be positive");
    double l = dmb::learned_train_body(c, radius, epochs, batch, lr, seed);
    if (loss_out) *loss_out = l;
    c->pc_valid = false;
  });
}

int dmb_net_param_count(void) { return dmb::net_param_count(); }

dmb_status dmb_net_get(dmb_ctx *c, float *w) {
  return guarded(c, [&] {
    DMB_REQUIRE(w, DMB_ERR_ARGUMENT, "weights output is NULL");
    dmb::net_get(c, w);
  });
}

dmb_status dmb_net_set(dmb_ctx *c, const float *w) {
  return guarded(c, [&] {
    DMB_REQUIRE(w, DMB_ERR_ARGUMENT, "weights are NULL");
    for (int i = 0; i < dmb::net_param_count(); i++)
      DMB_REQUIRE(std::isfinite(w[i]), DMB_ERR_ARGUMENT, "weights must be finite");
    dmb::net_set(c, w);
  });
}

dmb_status dmb_net_loss_grad(dmb_ctx *c, const float *feat, const float *tgt, const float *wgt, const int *cnt,
                             int64_t nrows, float *grad, float *loss) {
  return guarded(c, [&] {
    DMB_REQUIRE(feat && tgt && wgt && cnt && grad && loss && nrows >= 1, DMB_ERR_ARGUMENT, "bad arrays");
    for (int64_t i = 0; i < nrows; i++)
      DMB_REQUIRE(cnt[i] >= 1 && cnt[i] <= 64, DMB_ERR_ARGUMENT, "row sizes must be in 1..64");
    dmb::net_loss_grad(c, feat, tgt, wgt, cnt, nrows, grad, loss);
  });
}

dmb_status dmb_rhs_dipoles(dmb_ctx *c, int64_t R, const double *positions, const double *moments,
                           const int *magnetic, const double *frequencies, int quad_order, double *V_out) {
  return guarded(c, [&] {
    DMB_REQUIRE(c->have_rwg, DMB_ERR_STATE, "mesh and RWG data must be uploaded first");
    DMB_REQUIRE(R >= 1 && positions && moments && magnetic && frequencies && V_out, DMB_ERR_ARGUMENT,
                "bad dipole arrays");
    check_finite(positions, 3 * R, "dipole positions");
    check_finite(moments, 6 * R, "dipole moments");
    for (int64_t r = 0; r < R; r++) {
      DMB_REQUIRE(magnetic[r] == 0 || magnetic[r] == 1, DMB_ERR_ARGUMENT,
                  "Dipole type must be :electric or :magnetic");
      DMB_REQUIRE(std::isfinite(frequencies[r]) && frequencies[r] > 0, DMB_ERR_ARGUMENT,
                  "dipole frequency must be finite and positive");
    }
    const size_t bytes = sizeof(double2) * c->n * R;
    DevBuf bv;
    bv.ensure(bytes);
    dmb::rhs_dipoles_dev(c, R, positions, moments, magnetic, frequencies, quad_order, bv.as<double>());
    DMB_CUDA(cudaMemcpyAsync(V_out, bv.p, bytes, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
  });
}

dmb_status dmb_rhs_pattern_feed(dmb_ctx *c, int ntheta, const double *theta, int nphi, const double *phi,
                                const double *Ftheta, const double *Fphi, double frequency,
                                const double *phase_center, int conj_convention, int quad_order, double *V_out) {
  return guarded(c, [&] {
    DMB_REQUIRE(c->have_rwg, DMB_ERR_STATE, "mesh and RWG data must be uploaded first");
    DMB_REQUIRE(theta && phi && Ftheta && Fphi && phase_center && V_out, DMB_ERR_ARGUMENT, "bad pattern arrays");
    DMB_REQUIRE(ntheta >= 2, DMB_ERR_ARGUMENT, "Pattern feed requires at least 2 theta samples.");
    DMB_REQUIRE(nphi >= 2, DMB_ERR_ARGUMENT, "Pattern feed requires at least 2 phi samples.");
    check_finite(theta, ntheta, "Theta grid");
    check_finite(phi, nphi, "Phi grid");
    for (int i = 1; i < ntheta; i++)
      DMB_REQUIRE(theta[i] > theta[i - 1], DMB_ERR_ARGUMENT, "Theta grid must be strictly increasing.");
    for (int i = 1; i < nphi; i++)
      DMB_REQUIRE(phi[i] > phi[i - 1], DMB_ERR_ARGUMENT, "Phi grid must be strictly increasing.");
    DMB_REQUIRE(theta[0] >= -1e-12 && theta[ntheta - 1] <= 3.14159265358979323846 + 1e-12, DMB_ERR_ARGUMENT,
                "Theta grid must lie in [0, pi] (radians).");
    const double span = phi[nphi - 1] - phi[0];
    DMB_REQUIRE(span > 0 && span < 2.0 * 3.14159265358979323846 - 1e-12, DMB_ERR_ARGUMENT,
                "Phi grid should cover one open 2 pi period without a duplicate endpoint.");
    check_finite(Ftheta, 2 * (int64_t)ntheta * nphi, "pattern Ftheta");
    check_finite(Fphi, 2 * (int64_t)ntheta * nphi, "pattern Fphi");
    check_finite(phase_center, 3, "pattern phase_center");
    DMB_REQUIRE(std::isfinite(frequency) && frequency > 0, DMB_ERR_ARGUMENT,
                "Pattern feed frequency must be finite and positive.");
    const size_t bytes = sizeof(double2) * c->n;
    DevBuf bv;
    bv.ensure(bytes);
    dmb::rhs_pattern_dev(c, ntheta, theta, nphi, phi, Ftheta, Fphi, frequency, phase_center,
                         conj_convention ? 1 : 0, quad_order, bv.as<double>());
    DMB_CUDA(cudaMemcpyAsync(V_out, bv.p, bytes, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
  });
}

dmb_status dmb_gradient_impedance(dmb_ctx *c, int64_t R, const double *I, const double *lambda,
                                  const int *tri_patch, int64_t P, int reactive, int quad_order, double *g_out) {
  return guarded(c, [&] {
    DMB_REQUIRE(c->have_rwg, DMB_ERR_STATE, "mesh and RWG data must be uploaded first");
    DMB_REQUIRE(R >= 1 && I && lambda && tri_patch && g_out && P >= 0, DMB_ERR_ARGUMENT,
                "bad gradient arguments");
    DMB_REQUIRE(P <= 65535 && R <= 65535, DMB_ERR_ARGUMENT, "at most 65,535 patches and columns per call");
    for (int64_t t = 0; t < c->nt; t++)
      DMB_REQUIRE(tri_patch[t] >= 0 && tri_patch[t] < P, DMB_ERR_ARGUMENT,
                  "partition.tri_patch entries must lie in 0..P-1");
    check_finite(I, 2 * c->n * R, "I must contain only finite values");
    check_finite(lambda, 2 * c->n * R, "lambda must contain only finite values");
    if (P == 0) return;
    const size_t vb = sizeof(double2) * c->n * R;
    DevBuf bi, bl, bg;
    bi.ensure(vb);
    bl.ensure(vb);
    bg.ensure(sizeof(double) * P * R);
    DMB_CUDA(cudaMemcpyAsync(bi.p, I, vb, cudaMemcpyHostToDevice, c->stream));
    DMB_CUDA(cudaMemcpyAsync(bl.p, lambda, vb, cudaMemcpyHostToDevice, c->stream));
    dmb::gradient_impedance_dev(c, R, bi.as<double2>(), bl.as<double2>(), tri_patch, P, reactive ? 1 : 0,
                                quad_order, bg.as<double>());
    DMB_CUDA(cudaMemcpyAsync(g_out, bg.p, sizeof(double) * P * R, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
  });
}

dmb_status dmb_rhs_plane_waves(dmb_ctx *c, const double *kvecs, const double *E0s, const double *pols,
                               int64_t R, int quad_order, double *V_out) {
  return guarded(c, [&] {
    DMB_REQUIRE(kvecs && E0s && pols && V_out && R >= 1, DMB_ERR_ARGUMENT, "bad plane-wave arrays");
    check_finite(kvecs, 3 * R, "plane-wave k_vec");
    check_finite(E0s, R, "plane-wave amplitude E0");
    check_finite(pols, 3 * R, "plane-wave polarization");
    for (int64_t r = 0; r < R; r++) {
      const double *kv = kvecs + 3 * r, *pl = pols + 3 * r;
      double kn = std::sqrt(kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2]);
      double pn = std::sqrt(pl[0] * pl[0] + pl[1] * pl[1] + pl[2] * pl[2]);
      DMB_REQUIRE(kn > 0, DMB_ERR_ARGUMENT, "plane-wave k_vec must have a finite, nonzero norm.");
      DMB_REQUIRE(std::fabs(pn - 1.0) <= 1e-10 * std::max(1.0, pn) + 1e-12, DMB_ERR_ARGUMENT,
                  "plane-wave polarization must be a unit vector");
      double dt = std::fabs((kv[0] * pl[0] + kv[1] * pl[1] + kv[2] * pl[2]) / (kn * pn));
      DMB_REQUIRE(dt <= 1e-10, DMB_ERR_ARGUMENT, "plane-wave polarization must be transverse to k_vec");
    }
    size_t bytes = sizeof(double2) * c->n * R;
    DevBuf bv;
    bv.ensure(bytes);
    dmb::rhs_plane_waves_dev(c, kvecs, E0s, pols, R, quad_order, bv.as<double>());
    DMB_CUDA(cudaMemcpyAsync(V_out, bv.p, bytes, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
  });
}

dmb_status dmb_gmres(dmb_ctx *c, const double *rhs, double *x, int64_t nrhs, double tol, int maxiter,
                     int precond_kind, int precond_side, int check_convergence,
                     dmb_gmres_stats *stats) {
  dmb_gmres_stats st{};
  dmb_status s = guarded(c, [&] {
    DMB_REQUIRE(std::isfinite(tol) && tol > 0, DMB_ERR_ARGUMENT, "GMRES tol must be finite and positive");
    DMB_REQUIRE(maxiter >= 1, DMB_ERR_ARGUMENT, "GMRES maxiter must be at least 1");
    DMB_REQUIRE(precond_side == DMB_SIDE_LEFT || precond_side == DMB_SIDE_RIGHT, DMB_ERR_ARGUMENT,
                "Invalid precond_side (expected :left or :right)");
    DMB_REQUIRE(rhs && x && nrhs >= 1, DMB_ERR_ARGUMENT, "bad GMRES arrays");
    DMB_REQUIRE(dmb::operator_ready(c), DMB_ERR_STATE, "no assembled impedance matrix");
    check_finite(rhs, 2 * c->n * nrhs, "right-hand side");
    size_t bytes = sizeof(double2) * c->n * nrhs;
    DevBuf bb, bx;
    bb.ensure(bytes);
    bx.ensure(bytes);
    DMB_CUDA(cudaMemcpyAsync(bb.p, rhs, bytes, cudaMemcpyHostToDevice, c->stream));
    dmb::gmres_dev(c, bb.as<double>(), bx.as<double>(), nrhs, tol, maxiter, precond_kind,
                   precond_side, &st);
    DMB_CUDA(cudaMemcpyAsync(x, bx.p, bytes, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
    if (check_convergence && !st.solved)
      throw DmbError{DMB_ERR_NOT_CONVERGED,
                     "forward GMRES did not converge consistently: niter=" + std::to_string(st.niter) +
                         ", final_residual=" + std::to_string(st.residual) +
                         ", tol=" + std::to_string(tol) + ", maxiter=" + std::to_string(maxiter)};
  });
  if (stats) *stats = st;
  return s;
}

dmb_status dmb_gmres_adjoint(dmb_ctx *c, const double *rhs, double *x, int64_t nrhs, double tol, int maxiter,
                             int precond_kind, int precond_side, int check_convergence, dmb_gmres_stats *stats) {
  dmb_gmres_stats st{};
  dmb_status s = guarded(c, [&] {
    DMB_REQUIRE(std::isfinite(tol) && tol > 0, DMB_ERR_ARGUMENT, "GMRES tol must be finite and positive");
    DMB_REQUIRE(maxiter >= 1, DMB_ERR_ARGUMENT, "GMRES maxiter must be at least 1");
    DMB_REQUIRE(precond_side == DMB_SIDE_LEFT || precond_side == DMB_SIDE_RIGHT, DMB_ERR_ARGUMENT,
                "Invalid precond_side (expected :left or :right)");
    DMB_REQUIRE(precond_kind == DMB_PRECOND_NONE || precond_kind == DMB_PRECOND_NF_LU ||
                    precond_kind == DMB_PRECOND_NF_DIAG,
                DMB_ERR_ARGUMENT, "adjoint GMRES takes no preconditioner or a near-field one");
    DMB_REQUIRE(rhs && x && nrhs >= 1, DMB_ERR_ARGUMENT, "bad GMRES arrays");
    DMB_REQUIRE(dmb::operator_ready(c), DMB_ERR_STATE, "no assembled impedance matrix");
    check_finite(rhs, 2 * c->n * nrhs, "right-hand side");
    const int64_t cnt = c->n * nrhs;
    size_t bytes = sizeof(double2) * cnt;
    DevBuf bb, bx;
    bb.ensure(bytes);
    bx.ensure(bytes);
    DMB_CUDA(cudaMemcpyAsync(bb.p, rhs, bytes, cudaMemcpyHostToDevice, c->stream));
    // Z and the near-field matrix are complex symmetric: Z^H x = b  <=>
    // Z conj(x) = conj(b), and the adjoint preconditioner is conj(M^-1).  An
    // H-matrix A is not exactly symmetric: the same transformation gives
    // A^T conj(x) = conj(b), so its products run transposed meanwhile.
    dmb::conj_dev(c, bb.as<double2>(), cnt);
    struct Transposed {
      dmb_ctx *c;
      explicit Transposed(dmb_ctx *ctx) : c(ctx) { c->aca_transposed = c->op_kind == 1; }
      ~Transposed() { c->aca_transposed = false; }
    } tr(c);
    dmb::gmres_dev(c, bb.as<double>(), bx.as<double>(), nrhs, tol, maxiter, precond_kind, precond_side, &st);
    dmb::conj_dev(c, bx.as<double2>(), cnt);
    DMB_CUDA(cudaMemcpyAsync(x, bx.p, bytes, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
    if (check_convergence && !st.solved)
      throw DmbError{DMB_ERR_NOT_CONVERGED,
                     "adjoint GMRES did not converge consistently: niter=" + std::to_string(st.niter) +
                         ", final_residual=" + std::to_string(st.residual) +
                         ", tol=" + std::to_string(tol) + ", maxiter=" + std::to_string(maxiter)};
  });
  if (stats) *stats = st;
  return s;
}

dmb_status dmb_solve_direct(dmb_ctx *c, const double *rhs, double *x, int64_t nrhs,
                            double *backward_error_out) {
  return guarded(c, [&] {
    DMB_REQUIRE(rhs && x && nrhs >= 1, DMB_ERR_ARGUMENT, "bad solve arrays");
    DMB_REQUIRE(c->z_valid && c->op_kind == 0, DMB_ERR_STATE, "no assembled impedance matrix");
    check_finite(rhs, 2 * c->n * nrhs, "right-hand side");
    size_t bytes = sizeof(double2) * c->n * nrhs;
    DevBuf bb, bx;
    bb.ensure(bytes);
    bx.ensure(bytes);
    DMB_CUDA(cudaMemcpyAsync(bb.p, rhs, bytes, cudaMemcpyHostToDevice, c->stream));
    double berr = 0;
    dmb::solve_direct_dev(c, bb.as<double>(), bx.as<double>(), nrhs, &berr);
    DMB_CUDA(cudaMemcpyAsync(x, bx.p, bytes, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
    if (backward_error_out) *backward_error_out = berr;
  });
}

namespace {
void check_solve_params(const dmb_solve_params *p) {
  DMB_REQUIRE(p, DMB_ERR_ARGUMENT, "solve parameters are NULL");
  DMB_REQUIRE(std::isfinite(p->tol) && p->tol > 0, DMB_ERR_ARGUMENT, "GMRES tol must be finite and positive");
  DMB_REQUIRE(p->maxiter >= 1, DMB_ERR_ARGUMENT, "GMRES maxiter must be at least 1");
}

// assemble (+ surface impedance) + preconditioner of the resident solves
void resident_precond(dmb_ctx *c, const dmb_solve_params *p);

void resident_setup(dmb_ctx *c, const dmb_solve_params *p, const double *zs = nullptr) {
  dmb::assemble(c, p->k, p->eta0, p->quad_order, p->precision);
  if (zs) {
    check_finite(zs, 2 * c->nt, "surface impedance");
    dmb::apply_impedance(c, zs);
  }
  resident_precond(c, p);
}

// the auxiliary stream starts after everything issued so far on the context
// stream; aux_join orders the context stream after the auxiliary work
void aux_fork(dmb_ctx *c) {
  if (!c->stream_aux) {
    int least = 0, greatest = 0;
    DMB_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    DMB_CUDA(cudaStreamCreateWithPriority(&c->stream_aux, cudaStreamNonBlocking, least));
  }
  for (auto &e : c->aux_ev)
    if (!e) DMB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  DMB_CUDA(cudaEventRecord(c->aux_ev[0], c->stream));
  DMB_CUDA(cudaStreamWaitEvent(c->stream_aux, c->aux_ev[0], 0));
}

void aux_join(dmb_ctx *c) {
  DMB_CUDA(cudaEventRecord(c->aux_ev[1], c->stream_aux));
  DMB_CUDA(cudaStreamWaitEvent(c->stream, c->aux_ev[1], 0));
}

void resident_precond(dmb_ctx *c, const dmb_solve_params *p) {
  if (p->precond_kind == DMB_PRECOND_NF_LU || p->precond_kind == DMB_PRECOND_NF_DIAG) {
    DMB_REQUIRE(!std::isnan(p->cutoff) && p->cutoff >= 0, DMB_ERR_ARGUMENT,
                "near-field cutoff must be nonnegative and not NaN");
    dmb::nf_build(c, p->cutoff, p->precond_kind);
  } else if (p->precond_kind == DMB_PRECOND_LOCAL_INV) {
    dmb::local_inverse_build(c, p->cutoff, 64);
  } else if (p->precond_kind == DMB_PRECOND_RING) {
    dmb::ring_step_build(c, p->cutoff, false);
  } else if (p->precond_kind == DMB_PRECOND_LEARNED) {
    dmb::learned_build(c, p->cutoff);
  }
}

void resident_check(const dmb_gmres_stats &st) {
  if (!st.solved)
    throw DmbError{DMB_ERR_NOT_CONVERGED, "forward GMRES did not converge: niter=" + std::to_string(st.niter) +
                                              ", final_residual=" + std::to_string(st.residual)};
}
}  // namespace

dmb_status dmb_solve_resident(dmb_ctx *c, const dmb_solve_params *p, dmb_gmres_stats *stats) {
  dmb_gmres_stats st{};
  dmb_status s = guarded(c, [&] {
    check_solve_params(p);
    check_finite(p->kvec, 3, "plane-wave k_vec");
    check_finite(p->pol, 3, "plane-wave polarization");
    double t0 = dmb::now_ms();
    PcBf16Scope bf_scope(c);
    resident_setup(c, p);
    size_t bytes = sizeof(double2) * c->n;
    c->d_rhs.ensure(bytes);
    c->d_sol.ensure(bytes);
    c->sol_r = 0;
    dmb::rhs_plane_waves_dev(c, p->kvec, &p->E0, p->pol, 1, p->quad_order, c->d_rhs.as<double>());
    dmb::gmres_dev(c, c->d_rhs.as<double>(), c->d_sol.as<double>(), 1, p->tol, p->maxiter, p->precond_kind,
                   p->precond_side, &st);
    c->sol_r = 1;
    c->tm.solve_ms = dmb::now_ms() - t0;
    resident_check(st);
  });
  if (stats) *stats = st;
  return s;
}

dmb_status dmb_solve_resident_many(dmb_ctx *c, const dmb_solve_params *p, int64_t R, const double *kvecs,
                                   const double *E0s, const double *pols, double *sigma_out,
                                   dmb_gmres_stats *stats) {
  dmb_gmres_stats st{};
  dmb_status s = guarded(c, [&] {
    check_solve_params(p);
    DMB_REQUIRE(R >= 1 && kvecs && E0s && pols, DMB_ERR_ARGUMENT, "need R >= 1 incidences with k_vec, E0, pol");
    check_finite(kvecs, 3 * R, "plane-wave k_vecs");
    check_finite(pols, 3 * R, "plane-wave polarizations");
    check_finite(E0s, R, "plane-wave amplitudes");
    for (int64_t r = 0; r < R; r++) {
      const double *kv = kvecs + 3 * r;
      DMB_REQUIRE(kv[0] != 0.0 || kv[1] != 0.0 || kv[2] != 0.0, DMB_ERR_ARGUMENT, "plane-wave k_vec is zero");
      DMB_REQUIRE(E0s[r] != 0.0 || !sigma_out, DMB_ERR_ARGUMENT, "RCS needs a nonzero incident amplitude");
    }
    double t0 = dmb::now_ms();
    PcBf16Scope bf_scope(c);
    dmb::assemble(c, p->k, p->eta0, p->quad_order, p->precision);
    const size_t bytes = sizeof(double2) * c->n * R;
    c->d_rhs.ensure(bytes);
    c->d_sol.ensure(bytes);
    c->sol_r = 0;
    // the right-hand sides and the int8 slices of Z need only Z and the mesh:
    // they run on the auxiliary stream beside the preconditioner build
    aux_fork(c);
    {
      StreamSwap sw(c, c->stream_aux);
      dmb::rhs_plane_waves_async(c, kvecs, E0s, pols, R, p->quad_order, c->d_rhs.as<double>());
      if (dmb::krylov_exact_int8(c, R)) dmb::oz_prepare(c);
    }
    resident_precond(c, p);
    aux_join(c);
    c->tm.rhs_ms = 0.0;  // overlapped with the preconditioner build
    dmb::gmres_dev(c, c->d_rhs.as<double>(), c->d_sol.as<double>(), R, p->tol, p->maxiter, p->precond_kind,
                   p->precond_side, &st);
    c->sol_r = R;
    if (sigma_out) {
      c->d_mono.ensure(sizeof(double2) * 3 * R + sizeof(double) * R);
      double *E = c->d_mono.as<double>();
      double *sig = E + 6 * R;
      dmb::monostatic_dev(c, R, p->k, p->eta0, p->quad_order, c->d_sol.as<double>(), E, sig);
      DMB_CUDA(cudaMemcpyAsync(sigma_out, sig, sizeof(double) * R, cudaMemcpyDeviceToHost, c->stream));
      DMB_CUDA(cudaStreamSynchronize(c->stream));
    }
    c->tm.solve_ms = dmb::now_ms() - t0;
    resident_check(st);
  });
  if (stats) *stats = st;
  return s;
}

dmb_status dmb_copy_solution(dmb_ctx *c, double *I_out) {
  return guarded(c, [&] {
    DMB_REQUIRE(I_out && c->d_sol.p && c->sol_r > 0, DMB_ERR_STATE, "no resident solution");
    DMB_CUDA(cudaMemcpyAsync(I_out, c->d_sol.p, sizeof(double2) * c->n * c->sol_r, cudaMemcpyDeviceToHost,
                             c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
  });
}

dmb_status dmb_get_stream(dmb_ctx *c, void **stream_out) {
  return guarded(c, [&] {
    DMB_REQUIRE(stream_out, DMB_ERR_ARGUMENT, "stream output is NULL");
    *stream_out = (void *)c->stream;
  });
}

dmb_status dmb_set_kernel_timing(dmb_ctx *c, int enable) {
  return guarded(c, [&] {
    kt_collect(c);
    while (enable && c->kt_pool.size() < 4096) {
      cudaEvent_t e;
      DMB_CUDA(cudaEventCreate(&e));
      c->kt_pool.push_back(e);
    }
    c->kt_enabled = enable != 0;
    for (int f = 0; f < dmb_ctx::KT_FAMILIES; f++) {
      c->kt_ms[f] = 0;
      c->kt_flops[f] = 0;
      c->kt_launches[f] = 0;
    }
  });
}

dmb_status dmb_kernel_timing(dmb_ctx *c, double *ms, int64_t *launches, double *flops) {
  return dmb_kernel_timing_family(c, 0, ms, launches, flops);
}

dmb_status dmb_kernel_timing_family(dmb_ctx *c, int family, double *ms, int64_t *launches, double *work) {
  return guarded(c, [&] {
    DMB_REQUIRE(family >= 0 && family < dmb_ctx::KT_FAMILIES, DMB_ERR_ARGUMENT, "kernel family must be 0 to 5");
    kt_collect(c);
    if (ms) *ms = c->kt_ms[family];
    if (launches) *launches = c->kt_launches[family];
    if (work) *work = c->kt_flops[family];
  });
}

dmb_status dmb_farfield(dmb_ctx *c, const double *rhat, int64_t NO, double k, double eta0,
                        int quad_order, const double *I, int64_t nrhs, double *E_out) {
  return guarded(c, [&] {
    DMB_REQUIRE(rhat && I && E_out && NO >= 1 && nrhs >= 1, DMB_ERR_ARGUMENT, "bad far-field arrays");
    DMB_REQUIRE(std::isfinite(k) && k > 0 && std::isfinite(eta0), DMB_ERR_ARGUMENT,
                "far-field wavenumber and eta0 must be finite");
    check_finite(rhat, 3 * NO, "far-field directions");
    check_finite(I, 2 * c->n * nrhs, "current coefficients");
    size_t ib = sizeof(double2) * c->n * nrhs, eb = sizeof(double2) * 3 * NO * nrhs;
    DevBuf bi, be;
    bi.ensure(ib);
    be.ensure(eb);
    DMB_CUDA(cudaMemcpyAsync(bi.p, I, ib, cudaMemcpyHostToDevice, c->stream));
    dmb::farfield_dev(c, rhat, NO, k, eta0, quad_order, bi.as<double>(), nrhs, be.as<double>());
    DMB_CUDA(cudaMemcpyAsync(E_out, be.p, eb, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
  });
}

// ---- batches of independent surfaces -----------------------------------
// One context per surface of a call (kept and reused by later calls: their
// buffers only grow), so every surface's Z can be assembled by the same
// launches; `lanes` host threads then run the per-surface stages.
struct dmb_batch {
  int device = 0;
  int lanes = 1;
  std::vector<dmb_ctx *> slots;
  dmb::BatchAsmBufs asm_bufs;
  cudaStream_t stream = nullptr;  // the batch-wide launches
  double last_assembly_ms = 0;
  std::string err;
};

dmb_status dmb_batch_create(int device, int lanes, dmb_batch **out) {
  if (!out || lanes < 1 || lanes > 64) return DMB_ERR_ARGUMENT;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return DMB_ERR_CUDA;
  auto *b = new dmb_batch();
  b->device = device;
  b->lanes = lanes;
  int least = 0, greatest = 0;
  if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess ||
      cudaStreamCreateWithPriority(&b->stream, cudaStreamNonBlocking, greatest) != cudaSuccess) {
    delete b;
    return DMB_ERR_CUDA;
  }
  *out = b;
  return DMB_OK;
}

dmb_status dmb_batch_destroy(dmb_batch *b) {
  if (!b) return DMB_OK;
  cudaSetDevice(b->device);
  for (dmb_ctx *c : b->slots) dmb_ctx_destroy(c);
  b->asm_bufs.far_jobs.release();
  b->asm_bufs.far_tasks.release();
  b->asm_bufs.far_err.release();
  b->asm_bufs.near_jobs.release();
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return DMB_OK;
}

const char *dmb_batch_last_error(const dmb_batch *b) { return b ? b->err.c_str() : "null batch"; }

dmb_status dmb_batch_assembly_ms(const dmb_batch *b, double *ms_out) {
  if (!b || !ms_out) return DMB_ERR_ARGUMENT;
  *ms_out = b->last_assembly_ms;
  return DMB_OK;
}

namespace {
// the stages of one surface after the batch-wide assembly: impedance
// loading, preconditioner, RHS, GMRES, monostatic sigma; device times from
// events on the surface's stream (started after the assembly)
dmb_status batch_item(dmb_ctx *c, const dmb_solve_params *p, dmb_batch_item &it, cudaEvent_t ev_start,
                      cudaEvent_t ev_asm) {
  return guarded(c, [&] {
    cudaEvent_t e0, e1;
    DMB_CUDA(cudaEventCreate(&e0));
    DMB_CUDA(cudaEventCreate(&e1));
    DMB_CUDA(cudaStreamWaitEvent(c->stream, ev_asm, 0));
    DMB_CUDA(cudaEventRecord(e0, c->stream));
    PcBf16Scope bf_scope(c);
    if (it.zs) {
      check_finite(it.zs, 2 * c->nt, "surface impedance");
      dmb::apply_impedance(c, it.zs);
    }
    resident_precond(c, p);
    const size_t bytes = sizeof(double2) * c->n;
    c->d_rhs.ensure(bytes);
    c->d_sol.ensure(bytes);
    c->sol_r = 0;
    dmb::rhs_plane_waves_dev(c, it.kvec, &it.E0, it.pol, 1, p->quad_order, c->d_rhs.as<double>());
    dmb_gmres_stats gs{};
    dmb::gmres_dev(c, c->d_rhs.as<double>(), c->d_sol.as<double>(), 1, p->tol, p->maxiter, p->precond_kind,
                   p->precond_side, &gs);
    c->sol_r = 1;
    c->d_mono.ensure(sizeof(double2) * 3 + sizeof(double));
    double *E = c->d_mono.as<double>();
    dmb::monostatic_dev(c, 1, p->k, p->eta0, p->quad_order, c->d_sol.as<double>(), E, E + 6);
    DMB_CUDA(cudaMemcpyAsync(&it.sigma, E + 6, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (it.I_out)
      DMB_CUDA(cudaMemcpyAsync(it.I_out, c->d_sol.p, bytes, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaEventRecord(e1, c->stream));
    DMB_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    DMB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    it.solve_ms = ms;
    DMB_CUDA(cudaEventElapsedTime(&ms, ev_start, e1));
    it.latency_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    it.stats = gs;
    resident_check(gs);
  });
}

// run fn(i) for i in [0, count) on `lanes` host threads (items in the given
// order); the first failure stops the others and is reported
dmb_status lanes_run(dmb_batch *b, int64_t count, const std::vector<int64_t> &order,
                     const std::function<dmb_status(int64_t)> &fn) {
  std::atomic<int64_t> next{0};
  std::atomic<int> failed{0};
  std::mutex emu;
  dmb_status first_code = DMB_OK;
  std::vector<std::thread> workers;
  const int L = (int)std::min<int64_t>(b->lanes, count);
  for (int l = 0; l < L; l++) {
    workers.emplace_back([&] {
      cudaSetDevice(b->device);
      while (!failed.load()) {
        const int64_t i = next.fetch_add(1);
        if (i >= count) break;
        const int64_t s = order[i];
        const dmb_status st = fn(s);
        if (st != DMB_OK) {
          std::lock_guard<std::mutex> lk(emu);
          if (first_code == DMB_OK) {
            first_code = st;
            b->err = "surface " + std::to_string(s) + ": " + b->slots[s]->err;
          }
          failed.store(1);
        }
      }
    });
  }
  for (auto &w : workers) w.join();
  return first_code;
}
}  // namespace

dmb_status dmb_batch_solve(dmb_batch *b, const dmb_solve_params *p, dmb_batch_item *items, int64_t count,
                           double *device_ms_out) {
  if (!b) return DMB_ERR_ARGUMENT;
  b->err.clear();
  auto fail = [&](dmb_status s, const std::string &m) {
    b->err = m;
    return s;
  };
  if (!p || !items || count < 1) return fail(DMB_ERR_ARGUMENT, "batch needs parameters and >= 1 surface");
  if (!(std::isfinite(p->tol) && p->tol > 0) || p->maxiter < 1)
    return fail(DMB_ERR_ARGUMENT, "GMRES tol must be finite and positive and maxiter >= 1");
  if (cudaSetDevice(b->device) != cudaSuccess) return fail(DMB_ERR_CUDA, "cudaSetDevice failed");
  while ((int64_t)b->slots.size() < count) {
    dmb_ctx *c = nullptr;
    const dmb_status st = dmb_ctx_create(b->device, &c);
    if (st != DMB_OK) return fail(st, "could not create a surface context");
    // surfaces of changing sizes regrow buffers, so captured GMRES graphs
    // would rarely be replayed: direct launches
    c->gmres_graphs = false;
    b->slots.push_back(c);
  }
  for (int64_t i = 0; i < count; i++) {
    const dmb_batch_item &it = items[i];
    for (const double *v : {it.kvec, it.pol})
      for (int d = 0; d < 3; d++)
        if (!std::isfinite(v[d])) return fail(DMB_ERR_ARGUMENT, "surface " + std::to_string(i) + ": plane-wave "
                                                                  "k_vec and polarization must be finite");
    if (!(std::isfinite(items[i].E0) && items[i].E0 != 0.0))
      return fail(DMB_ERR_ARGUMENT, "surface " + std::to_string(i) + ": plane-wave E0 must be finite, nonzero");
  }
  std::vector<int64_t> order(count);
  for (int64_t i = 0; i < count; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t c2) { return items[a].n > items[c2].n; });
  cudaEvent_t ev_start = nullptr, ev_asm = nullptr;
  cudaEventCreate(&ev_start);
  cudaEventCreate(&ev_asm);
  // the batch's device time starts here: it includes the surfaces' set-up
  cudaEventRecord(ev_start, b->stream);
  // 1. uploads, host topology, per-triangle caches and far-pair panels,
  // lanes in parallel (each surface on its own stream); the panels need the
  // tile width, known once the tuner has timed the largest surface's size
  // bucket (on a first call they are built in step 2 instead)
  const bool f64 = p->precision == DMB_PREC_FP64;
  int64_t nmax = 0;
  for (int64_t i = 0; i < count; i++) nmax = std::max<int64_t>(nmax, items[i].n);
  dmb_status st = lanes_run(b, count, order, [&](int64_t s) {
    dmb_ctx *c = b->slots[s];
    const dmb_batch_item &it = items[s];
    dmb_status r = dmb_mesh_upload(c, it.xyz, it.tri, it.nv, it.nt);
    if (r == DMB_OK)
      r = dmb_rwg_upload(c, it.n, it.tplus, it.tminus, it.evert, it.vplus_opp, it.vminus_opp, it.len,
                         it.area_plus, it.area_minus);
    if (r == DMB_OK)
      r = guarded(c, [&] {
        dmb::ensure_cache(c, p->quad_order);
        const int T = dmb::far_tile_width_known(c, nmax, f64);
        if (T > 0) dmb::far_panels(c, T, f64);
      });
    return r;
  });
  if (st != DMB_OK) {
    cudaEventDestroy(ev_start);
    cudaEventDestroy(ev_asm);
    return st;
  }
  // 2. every surface's impedance matrix: the far tiles of all surfaces in one
  // launch, their near values and near sums in one launch each
  std::vector<dmb_ctx *> cs(b->slots.begin(), b->slots.begin() + count);
  {
    dmb_ctx *c0 = cs[0];
    std::lock_guard<std::mutex> lk(c0->mu);
    try {
      StreamSwap sw(c0, b->stream);
      b->last_assembly_ms = dmb::assemble_batch(cs, p->k, p->eta0, p->quad_order, p->precision, b->asm_bufs);
      DMB_CUDA(cudaEventRecord(ev_asm, b->stream));
    } catch (const DmbError &e) {
      cudaEventDestroy(ev_start);
      cudaEventDestroy(ev_asm);
      return fail((dmb_status)e.code, "batched assembly: " + e.msg);
    }
  }
  // 3. the per-surface stages, largest surface first
  st = lanes_run(b, count, order, [&](int64_t s) { return batch_item(b->slots[s], p, items[s], ev_start, ev_asm); });
  double total = 0;
  for (int64_t i = 0; i < count; i++) total = std::max(total, items[i].latency_ms);
  cudaEventDestroy(ev_start);
  cudaEventDestroy(ev_asm);
  if (device_ms_out) *device_ms_out = total;
  return st;
}

}  // extern "C"
