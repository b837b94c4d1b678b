// dmb_zgemm64.cu -- FP64 complex GEMM on the FP64 pipe for the plain (complex128)
// path: the Z X products of block GMRES with a complex128 Z (the zgemv of
// Krylov.gmres, one column per incidence), the trailing updates of the
// complex128 LDL^T (NearFieldPreconditioner.jl:705-715 factors the same
// matrix with UMFPACK) and the panel updates of its many-column triangular
// sweeps (:1044-1047).
//
//   Y(m, r)  =  sum_k A(m, k) B(k, r)        (OP 0)
//   Y(m, r) -=  sum_k A(m, k) B(k, r)        (OP 1)
//
// A(m, k) = A[m lda + k] (ALAY 0) or A[k lda + m] (ALAY 1); B(k, r) =
// B[r ldb + k]; Y(m, r) = Y[r ldy + m] (YLAY 0, column-major) or
// Y[m ldy + r] (YLAY 1, row-major).  LOWER keeps only r <= m (the lower
// triangle of a trailing update whose rows and columns start at the same
// index); tiles entirely above it exit at once.
//
// B200 has no FP64 tcgen05 kind, so the product runs on the FP64 FMA pipe
// (64 FMA per clock per SM).  A 256-thread CTA owns a 128 x 64 complex tile;
// each thread holds 8 x 4 complex accumulators (64 doubles) and per k step
// loads 8 + 4 complex operands from shared memory for 128 FMAs.  The two
// threads of a warp that share a row group read the same A address
// (broadcast); the 16 column threads read 16 consecutive B entries.  K runs
// in chunks of 8 through two shared-memory stages filled by cp.async (padded
// rows: conflict-free stores from the coalesced global reads); the next chunk
// is in flight while the current one is consumed.
#include <algorithm>

#include "dmb_device.cuh"
#include "dmb_internal.h"

namespace {

constexpr int ZG_BM = 128, ZG_BN = 64, ZG_KC = 8;
constexpr int ZG_A_STAGE = ZG_KC * (ZG_BM + 1), ZG_B_STAGE = ZG_KC * (ZG_BN + 1);
constexpr size_t ZG_SMEM = sizeof(double2) * 2 * (ZG_A_STAGE + ZG_B_STAGE);  // two stages: 49,664 B

// 16-byte global -> shared copy; src_bytes 0 fills the destination with zeros
// (src is then a valid address that is not read)
__device__ __forceinline__ void cp16(void *dst, const void *src, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

template <int ALAY, int YLAY, int OP, bool LOWER>
__global__ void __launch_bounds__(256, 1) k_zgemm64(int64_t M, int64_t R, int64_t K, const double2 *A, int64_t lda,
                                                     const double2 *B, int64_t ldb, double2 *Y, int64_t ldy) {
  extern __shared__ __align__(16) double2 zg_smem[];
  const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
  const int64_t m0 = (int64_t)blockIdx.x * ZG_BM, n0 = (int64_t)blockIdx.y * ZG_BN;
  if (LOWER && n0 > m0 + ZG_BM - 1) return;
  // chunk c of K (KC entries) into stage s: four A and two B elements per thread
  auto issue = [&](int64_t k0, int s) {
    double2 *As = zg_smem + s * ZG_A_STAGE;
    double2 *Bs = zg_smem + 2 * ZG_A_STAGE + s * ZG_B_STAGE;
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int e = t + 256 * u;
      const int mm = ALAY == 0 ? e >> 3 : e & 127, kk = ALAY == 0 ? e & 7 : e >> 7;
      const int64_t m = m0 + mm, k = k0 + kk;
      const bool in = m < M && k < K;
      cp16(As + kk * (ZG_BM + 1) + mm, in ? (ALAY == 0 ? A + m * lda + k : A + k * lda + m) : A, in ? 16 : 0);
    }
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int e = t + 256 * u;
      const int rr = e >> 3, kk = e & 7;
      const int64_t r = n0 + rr, k = k0 + kk;
      const bool in = r < R && k < K;
      cp16(Bs + kk * (ZG_BN + 1) + rr, in ? B + r * ldb + k : B, in ? 16 : 0);
    }
  };
  double2 acc[8][4];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = make_double2(0, 0);
  const int64_t nch = (K + ZG_KC - 1) / ZG_KC;
  if (nch > 0) issue(0, 0);
  cp_commit();
  for (int64_t ch = 0; ch < nch; ch++) {
    if (ch + 1 < nch) issue((ch + 1) * ZG_KC, (int)((ch + 1) & 1));
    cp_commit();
    cp_wait_prev();  // chunk ch has landed (this thread's copies)
    __syncthreads();
    const double2 *As = zg_smem + (ch & 1) * ZG_A_STAGE;
    const double2 *Bs = zg_smem + 2 * ZG_A_STAGE + (ch & 1) * ZG_B_STAGE;
#pragma unroll
    for (int kk = 0; kk < ZG_KC; kk++) {
      double2 a[8], b[4];
#pragma unroll
      for (int i = 0; i < 8; i++) a[i] = As[kk * (ZG_BM + 1) + ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = Bs[kk * (ZG_BN + 1) + tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) cfma(acc[i][j], a[i], b[j]);
    }
    __syncthreads();  // stage ch & 1 is refilled by the next iteration's issue
  }
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int64_t m = m0 + ty + 16 * i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int64_t r = n0 + tx + 16 * j;
      if (r >= R || (LOWER && r > m)) continue;
      double2 *p = YLAY == 0 ? Y + r * ldy + m : Y + m * ldy + r;
      *p = OP == 0 ? acc[i][j] : csub(*p, acc[i][j]);
    }
  }
}

template <int ALAY, int YLAY, int OP, bool LOWER>
void launch(dmb_ctx *c, int64_t M, int64_t R, int64_t K, const double2 *A, int64_t lda, const double2 *B, int64_t ldb,
            double2 *Y, int64_t ldy) {
  if (M <= 0 || R <= 0) return;
  static bool attr = false;  // one instantiation per template: set once per process
  if (!attr) {
    DMB_CUDA(cudaFuncSetAttribute(k_zgemm64<ALAY, YLAY, OP, LOWER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)ZG_SMEM));
    attr = true;
  }
  dim3 g((unsigned)((M + ZG_BM - 1) / ZG_BM), (unsigned)((R + ZG_BN - 1) / ZG_BN));
  DMB_LAUNCH(c, (k_zgemm64<ALAY, YLAY, OP, LOWER>), g, 256, ZG_SMEM, M, R, K, A, lda, B, ldb, Y, ldy);
}

}  // namespace

namespace dmb {

// Z X and the sweep updates are timed as kernel family 4 (8 flops per
// complex MAC); the factor's updates are timed by their caller (family 2).
void zgemm64_zx(dmb_ctx *c, const double2 *Z, const double2 *X, double2 *Y, int64_t N, int64_t R) {
  kt_begin(c);
  launch<0, 0, 0, false>(c, N, R, N, Z, N, X, N, Y, N);  // K = N = 0 still writes Y = 0
  kt_end(c, 8.0 * (double)N * (double)N * (double)R, 4);
}

void zgemm64_sub(dmb_ctx *c, bool a_transposed, int64_t M, int64_t R, int64_t K, const double2 *A, int64_t lda,
                 const double2 *B, int64_t ldb, double2 *Y, int64_t ldy) {
  if (K <= 0) return;
  kt_begin(c);
  if (a_transposed)
    launch<1, 0, 1, false>(c, M, R, K, A, lda, B, ldb, Y, ldy);
  else
    launch<0, 0, 1, false>(c, M, R, K, A, lda, B, ldb, Y, ldy);
  kt_end(c, 8.0 * (double)M * (double)R * (double)K, 4);
}

void zgemm64_lower_update(dmb_ctx *c, int64_t M, int64_t C, int64_t K, const double2 *W, int64_t ldw,
                          const double2 *Lrows, int64_t ldl, double2 *F, int64_t ldf) {
  if (K <= 0) return;
  launch<0, 1, 1, true>(c, M, C, K, W, ldw, Lrows, ldl, F, ldf);
}

}  // namespace dmb
