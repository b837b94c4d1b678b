// dmb_tc.cu -- tensor-core (tcgen05, sm_100a) trailing update of the complex64
// near-field factorisation:  C -= W L^T  on the lower tiles of the trailing
// matrix, W = L21 D1 and L = L21 (both rows >= j0, 64 complex columns).
//
// Precision: 3xTF32.  Each FP32 value x is split into hi = tf32(x) and
// lo = tf32(x - hi); the product keeps hi*hi + hi*lo + lo*hi (~21-22 bit
// accurate per term, FP32 accumulation in TMEM).
//
// Complex as one real GEMM.  With A' = [[Wr, -Wi], [Wi, Wr]] (2M x 128) and
// B' = [Lr, Li] (N x 128), A' B'^T = [C_re; C_im].  The 3xTF32 split stacks
// along K:  A'' = [A'hi, A'hi, A'lo],  B'' = [B'hi, B'lo, B'hi],  K = 384.
// k_tc_pack writes A'' so that every 64 complex rows occupy 128 consecutive
// rows (64 real-part rows, then 64 imaginary-part rows): one M = 128 UMMA tile
// therefore holds both parts of 64 complex rows, and the epilogue writes
// interleaved complex64 directly.
//
// Kernel k_tc_syrk (one CTA = 4 warps per 64 x 256 complex output tile):
//   warp 0 / lane 0   TMA producer, 4-stage ring of 128-B-swizzled K chunks
//                     (A 128 x 32 floats, B 256 x 32 floats per stage);
//   warp 1 / lane 0   issues tcgen05.mma.cta_group::1.kind::tf32
//                     (M 128, N 256, K 8) into a 256-column TMEM accumulator,
//                     tcgen05.commit frees each stage and finally signals done;
//   all 4 warps       tcgen05.ld the accumulator (warp w owns lanes 32w..),
//                     stage through shared memory, C -= acc on c <= r.
// Each TMA load fills one CTA's shared memory; no clusters.  Every mbarrier wait is bounded: on expiry
// the kernel records an error bit, stops issuing, frees its TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>

#include "dmb_device.cuh"
#include "dmb_internal.h"
#include "dmb_tcgen05.cuh"

namespace {

using namespace dmb_tc;

constexpr int TC_BM = 128;                 // real rows per tile (64 complex rows)
constexpr int TC_BN = 256;                 // complex columns per tile
constexpr int TC_BK = 32;                  // floats per stage (one 128-B swizzle row)
constexpr int TC_K = 6 * 256;              // floats per 256-wide complex K block: 3 (split) x 2 (re/im) x 256
constexpr int TC_STAGES = 4;
constexpr int TC_A_STAGE = TC_BM * TC_BK * 4;  // 16 KB
constexpr int TC_B_STAGE = TC_BN * TC_BK * 4;  // 32 KB
constexpr int TC_SMEM = TC_STAGES * (TC_A_STAGE + TC_B_STAGE) + 1024 /*barriers*/ + 1024 /*align*/;
constexpr int TC_SMEM_128 = TC_STAGES * (TC_A_STAGE + TC_B_STAGE / 2) + 1024 + 1024;
// factor-update pipeline depth, picked by the autotuner per update shape:
// 4 stages with one CTA per SM, or 2 stages with two co-resident CTAs per SM
constexpr int tc_syrk_smem(int stages) { return stages * (TC_A_STAGE + TC_B_STAGE) + 1024 + 1024; }

// One tcgen05.mma (M 128, N = BN, 32 bytes of K) on TF32 operands (K 8) or,
// with BF, on BF16 operands (kind::f16, both operands BF16, K 16); FP32
// accumulation either way.
template <int BN, bool BF>
__device__ __forceinline__ void umma_op(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  constexpr uint32_t fmt = BF ? 1u : 2u;  // operand format: BF16 (kind::f16) / TF32 (kind::tf32)
  constexpr uint32_t idesc = (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(BN >> 3) << 17) |
                             ((uint32_t)(TC_BM >> 4) << 24);
  if constexpr (BF)
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
  else
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Split of an FP32 value into the two operand pieces of the three-product
// scheme: TF32 hi = tf32(x), lo = tf32(x - hi) (~21 bits), or BF16 hi =
// bf16(x), lo = bf16(x - hi) (~16 bits).
__device__ __forceinline__ void split_op(float x, float &hi, float &lo) {
  hi = tf32_rna(x);
  lo = tf32_rna(x - hi);
}
__device__ __forceinline__ void split_op(float x, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}
// the same from a double (the residual taken in double)
__device__ __forceinline__ void split_op_d(double x, float &hi, float &lo) {
  hi = tf32_rna((float)x);
  lo = tf32_rna((float)(x - (double)hi));
}
__device__ __forceinline__ void split_op_d(double x, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
  hi = __float2bfloat16_rn((float)x);
  lo = __float2bfloat16_rn((float)(x - (double)__bfloat162float(hi)));
}
__device__ __forceinline__ float neg_op(float v) { return -v; }
__device__ __forceinline__ __nv_bfloat16 neg_op(__nv_bfloat16 v) { return __hneg(v); }
template <bool BF> struct OpElem { typedef float T; };
template <> struct OpElem<true> { typedef __nv_bfloat16 T; };

// ---------------------------------------------------------------------------
// operand packing for the trailing update, rows m in [0, rest) relative to r0,
// complex K in blocks of 256 (block kb at floats 1536 kb of a row):
//   A'' real row (128*(m/64) + m%64):      [Wr_h, -Wi_h, Wr_h, -Wi_h, Wr_l, -Wi_l]
//   A'' imag row (128*(m/64) + 64 + m%64): [Wi_h,  Wr_h, Wi_h,  Wr_h, Wi_l,  Wr_l]
//   B'' row m (m < ncols):                 [Lr_h,  Li_h, Lr_l,  Li_l, Lr_h,  Li_h]
// with W[r0 + m][woff + k] (stride wstride) and L[r0 + m][jcol + k]; k >= K zero.
// grid (rest, Kpad / 256), 256 threads.
// ---------------------------------------------------------------------------
template <class E>
__global__ void k_tc_pack(int64_t rest, int64_t ncols, int64_t N, int64_t r0, int64_t jcol, int K, int64_t ld,
                          const float2 *__restrict__ F, const float2 *__restrict__ W, int wstride, int woff,
                          E *__restrict__ Ap, E *__restrict__ Bp) {
  const int64_t m = blockIdx.x;
  const int kb = blockIdx.y, kk = threadIdx.x, k = kb * 256 + kk;
  if (m >= rest) return;
  float2 w = make_float2(0.f, 0.f), l = make_float2(0.f, 0.f);
  if (k < K) {
    w = W[(r0 + m) * wstride + woff + k];
    if (m < ncols) l = F[(r0 + m) * N + jcol + k];
  }
  E wrh, wrl, wih, wil;
  split_op(w.x, wrh, wrl);
  split_op(w.y, wih, wil);
  int64_t bi = m / 64, r = m % 64;
  E *ar = Ap + (128 * bi + r) * ld + kb * 1536;
  E *ai = Ap + (128 * bi + 64 + r) * ld + kb * 1536;
  const int S = 256;
  ar[kk] = wrh; ar[S + kk] = neg_op(wih); ar[2 * S + kk] = wrh; ar[3 * S + kk] = neg_op(wih);
  ar[4 * S + kk] = wrl; ar[5 * S + kk] = neg_op(wil);
  ai[kk] = wih; ai[S + kk] = wrh;  ai[2 * S + kk] = wih; ai[3 * S + kk] = wrh;  ai[4 * S + kk] = wil; ai[5 * S + kk] = wrl;
  if (m < ncols) {
    E lrh, lrl, lih, lil;
    split_op(l.x, lrh, lrl);
    split_op(l.y, lih, lil);
    E *br = Bp + m * ld + kb * 1536;
    br[kk] = lrh; br[S + kk] = lih;  br[2 * S + kk] = lrl; br[3 * S + kk] = lil;  br[4 * S + kk] = lrh; br[5 * S + kk] = lih;
  }
}

// Packed K blocks hold 1536 elements per 256 complex K: segments [hi x hi |
// hi x lo | lo x hi] of 512 elements each.  A K chunk is one 128-byte swizzle
// row: 32 TF32 or 64 BF16 elements.  cpb = chunks streamed per block: 48 / 24
// (TF32 / BF16, all three products) or 16 / 8 (hi x hi only).
template <bool BF>
__device__ __forceinline__ int tc_kx(int kc, int cpb) { return (kc / cpb) * 1536 + (kc % cpb) * (BF ? 64 : 32); }

template <int STAGES, bool BF>
__global__ void __launch_bounds__(128, (STAGES <= 2 ? 2 : 1)) k_tc_syrk(const __grid_constant__ CUtensorMap tmA,
                                                    const __grid_constant__ CUtensorMap tmB, float2 *__restrict__ F,
                                                    int64_t N, int64_t j0, int64_t rest, int64_t c_hi, int nchunks,
                                                    int cpb, unsigned *err) {
  // grid.x walks row blocks fastest, so CTAs running together share the
  // column block's B operand in L2
  const int64_t row0 = (int64_t)blockIdx.x * 64;   // complex rows of the tile (relative to j0)
  const int64_t col0 = (int64_t)blockIdx.y * TC_BN;
  if (row0 >= rest || col0 > row0 + 63 || j0 + col0 >= c_hi) return;  // uniform: tile outside the update

  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char *gbase = smem_raw + (base - raw);
  const uint32_t sA = base;                                  // STAGES x 16 KB
  const uint32_t sB = base + STAGES * TC_A_STAGE;         // STAGES x 32 KB
  const uint32_t sBar = sB + STAGES * TC_B_STAGE;         // full[4], empty[4], done
  uint64_t *bar_ptr = reinterpret_cast<uint64_t *>(gbase + (sBar - base));
  volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(bar_ptr + 16);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(bar_ptr + 17);
  const uint32_t full0 = sBar, empty0 = sBar + 8 * STAGES, done = sBar + 16 * STAGES;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(const_cast<uint32_t *>(tmem_slot))),
                 "r"(TC_BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem_d = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // TMA producer
    for (int kc = 0; kc < nchunks; kc++) {
      const int s = kc % STAGES;
      if (kc >= STAGES && !mbar_wait(empty0 + 8 * s, ((kc / STAGES) - 1) & 1, err, abort_flag)) break;
      mbar_expect_tx(full0 + 8 * s, TC_A_STAGE + TC_B_STAGE);
      const int kx = tc_kx<BF>(kc, cpb);
      tma_load_2d(sA + s * TC_A_STAGE, &tmA, kx, (int)(2 * row0), full0 + 8 * s);
      tma_load_2d(sB + s * TC_B_STAGE, &tmB, kx, (int)col0, full0 + 8 * s);
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    bool ok = true;
    for (int kc = 0; kc < nchunks && ok; kc++) {
      const int s = kc % STAGES;
      if (!mbar_wait(full0 + 8 * s, (kc / STAGES) & 1, err, abort_flag)) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int k = 0; k < TC_BK / 8; k++) {
        const uint64_t ad = sw128_desc(sA + s * TC_A_STAGE + k * 32);
        const uint64_t bd = sw128_desc(sB + s * TC_B_STAGE + k * 32);
        umma_op<TC_BN, BF>(tmem_d, ad, bd, (kc > 0 || k > 0) ? 1u : 0u);
      }
      umma_commit(empty0 + 8 * s);
    }
    if (ok) umma_commit(done);
  }
  __syncwarp();

  // epilogue (the decision to write back is made uniformly for the CTA)
  const int have = __syncthreads_and(mbar_wait(done, 0, err, abort_flag) ? 1 : 0);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (have) {
    float *E = reinterpret_cast<float *>(gbase);  // 128 x 33 staging (pipeline buffers are idle now)
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    for (int cc = 0; cc < TC_BN / 32; cc++) {
      uint32_t v[32];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
            "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
            "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
            "=r"(v[30]), "=r"(v[31])
          : "r"(tmem_d + lane_base + (uint32_t)(cc * 32)));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      const int row = warp * 32 + lane;
#pragma unroll
      for (int q = 0; q < 32; q++) E[row * 33 + q] = __uint_as_float(v[q]);
      __syncthreads();
      // thread -> (complex row r = rr + 4i, column q); all 16 loads are
      // issued before any store so they are in flight together
      const int q = threadIdx.x & 31, rr = threadIdx.x >> 5;
      const int64_t gc = j0 + col0 + cc * 32 + q;
      float2 cv[16];
#pragma unroll
      for (int i = 0; i < 16; i++) {
        const int64_t gr = j0 + row0 + rr + 4 * i;
        cv[i] = (gr < N && gc < c_hi && gc <= gr) ? F[gr * N + gc] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int i = 0; i < 16; i++) {
        const int r = rr + 4 * i;
        const int64_t gr = j0 + row0 + r;
        if (gr < N && gc < c_hi && gc <= gr)
          F[gr * N + gc] = make_float2(cv[i].x - E[r * 33 + q], cv[i].y - E[(64 + r) * 33 + q]);
      }
      __syncthreads();
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_d), "r"(TC_BN) : "memory");
}

// Persistent form of k_tc_syrk (autotuner candidate): a grid of at most one
// CTA per SM walks the lower tiles of the update (column tile outer, row
// tiles inner, tiles above the diagonal never launched) with 6 warps:
//   warp 4 / lane 0   TMA producer over (tile, K chunk) into a 4-stage ring;
//   warp 5 / lane 0   tcgen05.mma (M 128, N 256, K 8) into one of two
//                     256-column TMEM accumulators, in turn, so the next tile
//                     accumulates while the last one drains;
//   warps 0-3         drain: tcgen05.ld, stage through shared memory,
//                     C -= acc on c <= r, release the accumulator.
// Same MMA sequence per tile as k_tc_syrk, so the same bits.  Every wait is
// bounded (error bit, abort flag, TMEM freed).
constexpr int TCP_STAGES = 4;
constexpr int TCP_E_BYTES = TC_BM * 33 * 4;
constexpr int TCP_SMEM = TCP_STAGES * (TC_A_STAGE + TC_B_STAGE) + TCP_E_BYTES + 256 + 1024;

__device__ __forceinline__ void tcp_tile(int64_t t, int nrt, int nct, int &rt, int &ct) {
  for (ct = 0; ct < nct; ct++) {
    const int64_t n = nrt - 4 * ct;
    if (n <= 0) break;
    if (t < n) {
      rt = (int)(4 * ct + t);
      return;
    }
    t -= n;
  }
  rt = -1;
}

__device__ __forceinline__ void tcp_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tcp_epi_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

template <bool BF>
__global__ void __launch_bounds__(192, 1) k_tc_syrk_p(const __grid_constant__ CUtensorMap tmA,
                                                      const __grid_constant__ CUtensorMap tmB, float2 *__restrict__ F,
                                                      int64_t N, int64_t j0, int64_t c_hi, int nchunks, int cpb,
                                                      int nrt, int nct, int64_t ntiles, unsigned *err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char *gbase = smem_raw + (base - raw);
  const uint32_t sA = base;
  const uint32_t sB = base + TCP_STAGES * TC_A_STAGE;
  float *E = reinterpret_cast<float *>(gbase + TCP_STAGES * (TC_A_STAGE + TC_B_STAGE));
  const uint32_t sBar = sB + TCP_STAGES * TC_B_STAGE + TCP_E_BYTES;
  uint64_t *bar_ptr = reinterpret_cast<uint64_t *>(gbase + (sBar - base));
  volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(bar_ptr + 16);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(bar_ptr + 17);
  volatile int *epi_ok = reinterpret_cast<volatile int *>(bar_ptr + 18);
  const uint32_t full0 = sBar, empty0 = sBar + 8 * TCP_STAGES, accf0 = sBar + 16 * TCP_STAGES, acce0 = accf0 + 16;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < TCP_STAGES; s++) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(accf0 + 8 * b, 1);
      mbar_init(acce0 + 8 * b, 1);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(const_cast<uint32_t *>(tmem_slot))),
                 "r"(2 * TC_BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem_d = *tmem_slot;

  if (warp == 4) {
    if (lane == 0) {
      long long t = 0;
      bool go = true;
      for (int64_t tile = blockIdx.x; tile < ntiles && go; tile += gridDim.x) {
        int rt, ct;
        tcp_tile(tile, nrt, nct, rt, ct);
        const int64_t row0 = (int64_t)rt * 64, col0 = (int64_t)ct * TC_BN;
        for (int kc = 0; kc < nchunks; kc++, t++) {
          const int s = (int)(t % TCP_STAGES);
          if (*abort_flag || (t >= TCP_STAGES &&
                              !mbar_wait(empty0 + 8 * s, (uint32_t)((t / TCP_STAGES) - 1) & 1u, err, abort_flag))) {
            go = false;
            break;
          }
          mbar_expect_tx(full0 + 8 * s, TC_A_STAGE + TC_B_STAGE);
          const int kx = tc_kx<BF>(kc, cpb);
          tma_load_2d(sA + s * TC_A_STAGE, &tmA, kx, (int)(2 * row0), full0 + 8 * s);
          tma_load_2d(sB + s * TC_B_STAGE, &tmB, kx, (int)col0, full0 + 8 * s);
        }
      }
    }
  } else if (warp == 5) {
    if (lane == 0) {
      long long t = 0;
      int i = 0;
      bool ok = true;
      for (int64_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, i++) {
        const int buf = i & 1;
        if (i >= 2 && !mbar_wait(acce0 + 8 * buf, (uint32_t)((i >> 1) - 1) & 1u, err, abort_flag)) {
          ok = false;
          break;
        }
        const uint32_t tmem_acc = tmem_d + (uint32_t)(buf * TC_BN);
        for (int kc = 0; kc < nchunks; kc++, t++) {
          const int s = (int)(t % TCP_STAGES);
          if (!mbar_wait(full0 + 8 * s, (uint32_t)(t / TCP_STAGES) & 1u, err, abort_flag)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
          for (int k = 0; k < TC_BK / 8; k++) {
            const uint64_t ad = sw128_desc(sA + s * TC_A_STAGE + k * 32);
            const uint64_t bd = sw128_desc(sB + s * TC_B_STAGE + k * 32);
            umma_op<TC_BN, BF>(tmem_acc, ad, bd, (kc > 0 || k > 0) ? 1u : 0u);
          }
          umma_commit(empty0 + 8 * s);
        }
        if (ok) umma_commit(accf0 + 8 * buf);
      }
    }
  } else {
    // drain warps 0-3 (warp w reads TMEM lanes 32w..32w+31)
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    int i = 0;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, i++) {
      const int buf = i & 1;
      int rt, ct;
      tcp_tile(tile, nrt, nct, rt, ct);
      const int64_t row0 = (int64_t)rt * 64, col0 = (int64_t)ct * TC_BN;
      const bool got = mbar_wait(accf0 + 8 * buf, (uint32_t)(i >> 1) & 1u, err, abort_flag);
      if (threadIdx.x == 0) *epi_ok = 1;
      tcp_epi_sync();
      if (!got) *epi_ok = 0;
      tcp_epi_sync();
      if (!*epi_ok) break;  // uniform over the drain warps
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t tmem_acc = tmem_d + (uint32_t)(buf * TC_BN);
      for (int cc = 0; cc < TC_BN / 32; cc++) {
        uint32_t v[32];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
              "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
              "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
              "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
            : "r"(tmem_acc + lane_base + (uint32_t)(cc * 32)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int row = warp * 32 + lane;
#pragma unroll
        for (int q = 0; q < 32; q++) E[row * 33 + q] = __uint_as_float(v[q]);
        tcp_epi_sync();
        const int q = threadIdx.x & 31, rr = threadIdx.x >> 5;
        const int64_t gc = j0 + col0 + cc * 32 + q;
        float2 cv[16];
#pragma unroll
        for (int r16 = 0; r16 < 16; r16++) {
          const int64_t gr = j0 + row0 + rr + 4 * r16;
          cv[r16] = (gr < N && gc < c_hi && gc <= gr) ? F[gr * N + gc] : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int r16 = 0; r16 < 16; r16++) {
          const int r = rr + 4 * r16;
          const int64_t gr = j0 + row0 + r;
          if (gr < N && gc < c_hi && gc <= gr)
            F[gr * N + gc] = make_float2(cv[r16].x - E[r * 33 + q], cv[r16].y - E[(64 + r) * 33 + q]);
        }
        tcp_epi_sync();
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      tcp_epi_sync();
      if (threadIdx.x == 0) tcp_arrive(acce0 + 8 * buf);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_d), "r"(2 * TC_BN) : "memory");
}

// ---------------------------------------------------------------------------
// General complex GEMM  Y (op)= A B^T  for many right-hand sides.
//
// A'' (2 Mpad rows) and B'' (Rpad rows) hold K'' = 6 Kpad floats per row in
// blocks of 256 complex K: block kb occupies floats [1536 kb, 1536 kb + 1536)
// with the six 256-wide segments of the layout above.  One CTA computes a
// 64 x 256 complex tile over all nchunks 32-float K chunks (same warp roles and
// bounded waits as k_tc_syrk); the output is complex128 column-major,
// Y[m + r ldy] = acc (mode 0) or -= acc (mode 1).  A tiles start at row
// a_row0 + 2 row0 and float column a_kx0 of the A'' map (sub-blocks of a
// matrix packed once), B tiles at column 0.  grid.x walks the column
// tiles fastest, so the CTAs that share an A row tile run together and read it
// from DRAM once.
// ---------------------------------------------------------------------------
// ROLE only names the launch site for profilers: 0 = Z X of the Krylov
// operator, 1 = triangular-solve GEMMs.  BN (256 or 128) is the tile width in
// complex columns: the 128-wide form doubles the CTAs of launches that would
// otherwise fill fewer than two waves.
template <int ROLE, int BN, bool BF>
__global__ void __launch_bounds__(128, 1) k_tc_gemm(const __grid_constant__ CUtensorMap tmA,
                                                    const __grid_constant__ CUtensorMap tmB, int a_row0, int a_kx0,
                                                    int nchunks, int cpb, int64_t M, int64_t Rv,
                                                    double2 *__restrict__ Y, int64_t ldy, int mode, int tri,
                                                    unsigned *err) {
  constexpr int B_STAGE = BN * TC_BK * 4;
  const int64_t col0 = (int64_t)blockIdx.x * BN;
  const int64_t row0 = (int64_t)blockIdx.y * 64;
  if (row0 >= M || col0 >= Rv) return;  // uniform
  // triangular A (tri 1: lower, A[m][k] = 0 for k > m; tri 2: upper): only the
  // 256-wide K blocks that meet this row tile's rows are streamed (cpb chunks each)
  int kc0 = 0, kc1 = nchunks;
  if (tri == 1) kc1 = min(nchunks, cpb * (int)((row0 + 64 + 255) / 256));
  else if (tri == 2) kc0 = cpb * (int)(row0 / 256);
  const int nk = kc1 - kc0;

  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char *gbase = smem_raw + (base - raw);
  const uint32_t sA = base;
  const uint32_t sB = base + TC_STAGES * TC_A_STAGE;
  const uint32_t sBar = sB + TC_STAGES * B_STAGE;
  uint64_t *bar_ptr = reinterpret_cast<uint64_t *>(gbase + (sBar - base));
  volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(bar_ptr + 16);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(bar_ptr + 17);
  const uint32_t full0 = sBar, empty0 = sBar + 8 * TC_STAGES, done = sBar + 16 * TC_STAGES;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < TC_STAGES; s++) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(const_cast<uint32_t *>(tmem_slot))),
                 "r"(BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem_d = *tmem_slot;

  if (warp == 0 && lane == 0) {
    for (int i = 0; i < nk; i++) {
      const int s = i % TC_STAGES, kc = kc0 + i;
      if (i >= TC_STAGES && !mbar_wait(empty0 + 8 * s, ((i / TC_STAGES) - 1) & 1, err, abort_flag)) break;
      mbar_expect_tx(full0 + 8 * s, TC_A_STAGE + B_STAGE);
      const int kx = tc_kx<BF>(kc, cpb);
      tma_load_2d(sA + s * TC_A_STAGE, &tmA, a_kx0 + kx, a_row0 + (int)(2 * row0), full0 + 8 * s);
      tma_load_2d(sB + s * B_STAGE, &tmB, kx, (int)col0, full0 + 8 * s);
    }
  } else if (warp == 1 && lane == 0) {
    bool ok = true;
    for (int i = 0; i < nk && ok; i++) {
      const int s = i % TC_STAGES;
      if (!mbar_wait(full0 + 8 * s, (i / TC_STAGES) & 1, err, abort_flag)) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int k = 0; k < TC_BK / 8; k++) {
        const uint64_t ad = sw128_desc(sA + s * TC_A_STAGE + k * 32);
        const uint64_t bd = sw128_desc(sB + s * B_STAGE + k * 32);
        umma_op<BN, BF>(tmem_d, ad, bd, (i > 0 || k > 0) ? 1u : 0u);
      }
      umma_commit(empty0 + 8 * s);
    }
    if (ok) umma_commit(done);
  }
  __syncwarp();

  const int have = __syncthreads_and(mbar_wait(done, 0, err, abort_flag) ? 1 : 0);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (have) {
    float *E = reinterpret_cast<float *>(gbase);  // 128 x 33 staging
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    const int rl = threadIdx.x & 63, qh = threadIdx.x >> 6;
    const int64_t gr = row0 + rl;
    for (int cc = 0; cc < BN / 32; cc++) {
      if (col0 + cc * 32 >= Rv) break;  // uniform
      uint32_t v[32];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
            "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
            "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
            "=r"(v[30]), "=r"(v[31])
          : "r"(tmem_d + lane_base + (uint32_t)(cc * 32)));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      const int row = warp * 32 + lane;
#pragma unroll
      for (int q = 0; q < 32; q++) E[row * 33 + q] = __uint_as_float(v[q]);
      __syncthreads();
      // thread -> complex row rl (consecutive threads: consecutive rows of a
      // column); for the subtracting form all 16 loads are issued before any
      // store so they are in flight together
      if (gr < M) {
        const int64_t gc0 = col0 + cc * 32 + qh;
        if (mode == 0) {
#pragma unroll
          for (int i = 0; i < 16; i++) {
            const int q = qh + 2 * i;
            if (gc0 + 2 * i < Rv) Y[(gc0 + 2 * i) * ldy + gr] = make_double2(E[rl * 33 + q], E[(64 + rl) * 33 + q]);
          }
        } else {
          double2 cv[16];
#pragma unroll
          for (int i = 0; i < 16; i++)
            cv[i] = (gc0 + 2 * i < Rv) ? __ldcs(Y + (gc0 + 2 * i) * ldy + gr) : make_double2(0, 0);
#pragma unroll
          for (int i = 0; i < 16; i++) {
            const int q = qh + 2 * i;
            if (gc0 + 2 * i < Rv)
              __stcs(Y + (gc0 + 2 * i) * ldy + gr,
                     make_double2(cv[i].x - E[rl * 33 + q], cv[i].y - E[(64 + rl) * 33 + q]));
          }
        }
      }
      __syncthreads();
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_d), "r"(BN) : "memory");
}

// Persistent form of k_tc_gemm (autotuner candidate): a grid of at most one
// CTA per SM walks the tiles (column tile fastest), 6 warps as in k_tc_syrk_p
// (producer, MMA issuer, 4 drain warps) with two TMEM accumulators, so a
// tile's epilogue (the read-modify-write of complex128 Y) overlaps the next
// tile's main loop.  Same MMA sequence per tile as k_tc_gemm: the same bits.
template <int BN, bool BF>
__global__ void __launch_bounds__(192, 1) k_tc_gemm_p(const __grid_constant__ CUtensorMap tmA,
                                                      const __grid_constant__ CUtensorMap tmB, int a_row0, int a_kx0,
                                                      int nchunks, int cpb, int64_t M, int64_t Rv,
                                                      double2 *__restrict__ Y, int64_t ldy, int mode, int tri,
                                                      int ntc, int64_t ntiles, unsigned *err) {
  constexpr int B_STAGE = BN * TC_BK * 4;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char *gbase = smem_raw + (base - raw);
  const uint32_t sA = base;
  const uint32_t sB = base + TCP_STAGES * TC_A_STAGE;
  float *E = reinterpret_cast<float *>(gbase + TCP_STAGES * (TC_A_STAGE + B_STAGE));
  const uint32_t sBar = sB + TCP_STAGES * B_STAGE + TCP_E_BYTES;
  uint64_t *bar_ptr = reinterpret_cast<uint64_t *>(gbase + (sBar - base));
  volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(bar_ptr + 16);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(bar_ptr + 17);
  volatile int *epi_ok = reinterpret_cast<volatile int *>(bar_ptr + 18);
  const uint32_t full0 = sBar, empty0 = sBar + 8 * TCP_STAGES, accf0 = sBar + 16 * TCP_STAGES, acce0 = accf0 + 16;
  // K chunk range of a row tile (triangular A: only the 256-wide K blocks
  // that meet the tile's rows)
  auto krange = [&](int64_t row0, int &kc0, int &kc1) {
    kc0 = 0;
    kc1 = nchunks;
    if (tri == 1) kc1 = min(nchunks, cpb * (int)((row0 + 64 + 255) / 256));
    else if (tri == 2) kc0 = cpb * (int)(row0 / 256);
  };

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < TCP_STAGES; s++) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(accf0 + 8 * b, 1);
      mbar_init(acce0 + 8 * b, 1);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(const_cast<uint32_t *>(tmem_slot))),
                 "r"(2 * BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem_d = *tmem_slot;

  if (warp == 4) {
    if (lane == 0) {
      long long t = 0;
      bool go = true;
      for (int64_t tile = blockIdx.x; tile < ntiles && go; tile += gridDim.x) {
        const int64_t row0 = (tile / ntc) * 64, col0 = (tile % ntc) * BN;
        int kc0, kc1;
        krange(row0, kc0, kc1);
        for (int kc = kc0; kc < kc1; kc++, t++) {
          const int s = (int)(t % TCP_STAGES);
          if (*abort_flag || (t >= TCP_STAGES &&
                              !mbar_wait(empty0 + 8 * s, (uint32_t)((t / TCP_STAGES) - 1) & 1u, err, abort_flag))) {
            go = false;
            break;
          }
          mbar_expect_tx(full0 + 8 * s, TC_A_STAGE + B_STAGE);
          const int kx = tc_kx<BF>(kc, cpb);
          tma_load_2d(sA + s * TC_A_STAGE, &tmA, a_kx0 + kx, a_row0 + (int)(2 * row0), full0 + 8 * s);
          tma_load_2d(sB + s * B_STAGE, &tmB, kx, (int)col0, full0 + 8 * s);
        }
      }
    }
  } else if (warp == 5) {
    if (lane == 0) {
      long long t = 0;
      int i = 0;
      bool ok = true;
      for (int64_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, i++) {
        const int64_t row0 = (tile / ntc) * 64;
        int kc0, kc1;
        krange(row0, kc0, kc1);
        const int buf = i & 1;
        if (i >= 2 && !mbar_wait(acce0 + 8 * buf, (uint32_t)((i >> 1) - 1) & 1u, err, abort_flag)) {
          ok = false;
          break;
        }
        const uint32_t tmem_acc = tmem_d + (uint32_t)(buf * BN);
        for (int kc = kc0; kc < kc1; kc++, t++) {
          const int s = (int)(t % TCP_STAGES);
          if (!mbar_wait(full0 + 8 * s, (uint32_t)(t / TCP_STAGES) & 1u, err, abort_flag)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
          for (int k = 0; k < TC_BK / 8; k++) {
            const uint64_t ad = sw128_desc(sA + s * TC_A_STAGE + k * 32);
            const uint64_t bd = sw128_desc(sB + s * B_STAGE + k * 32);
            umma_op<BN, BF>(tmem_acc, ad, bd, (kc > kc0 || k > 0) ? 1u : 0u);
          }
          umma_commit(empty0 + 8 * s);
        }
        if (ok) umma_commit(accf0 + 8 * buf);
      }
    }
  } else {
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    const int rl = threadIdx.x & 63, qh = threadIdx.x >> 6;
    int i = 0;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, i++) {
      const int buf = i & 1;
      const int64_t row0 = (tile / ntc) * 64, col0 = (tile % ntc) * BN;
      const bool got = mbar_wait(accf0 + 8 * buf, (uint32_t)(i >> 1) & 1u, err, abort_flag);
      if (threadIdx.x == 0) *epi_ok = 1;
      tcp_epi_sync();
      if (!got) *epi_ok = 0;
      tcp_epi_sync();
      if (!*epi_ok) break;  // uniform over the drain warps
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t tmem_acc = tmem_d + (uint32_t)(buf * BN);
      const int64_t gr = row0 + rl;
      for (int cc = 0; cc < BN / 32; cc++) {
        if (col0 + cc * 32 >= Rv) break;  // uniform
        uint32_t v[32];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
              "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
              "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
              "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
            : "r"(tmem_acc + lane_base + (uint32_t)(cc * 32)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int row = warp * 32 + lane;
#pragma unroll
        for (int q = 0; q < 32; q++) E[row * 33 + q] = __uint_as_float(v[q]);
        tcp_epi_sync();
        if (gr < M) {
          const int64_t gc0 = col0 + cc * 32 + qh;
          if (mode == 0) {
#pragma unroll
            for (int r16 = 0; r16 < 16; r16++) {
              const int q = qh + 2 * r16;
              if (gc0 + 2 * r16 < Rv)
                Y[(gc0 + 2 * r16) * ldy + gr] = make_double2(E[rl * 33 + q], E[(64 + rl) * 33 + q]);
            }
          } else {
            double2 cv[16];
#pragma unroll
            for (int r16 = 0; r16 < 16; r16++)
              cv[r16] = (gc0 + 2 * r16 < Rv) ? __ldcs(Y + (gc0 + 2 * r16) * ldy + gr) : make_double2(0, 0);
#pragma unroll
            for (int r16 = 0; r16 < 16; r16++) {
              const int q = qh + 2 * r16;
              if (gc0 + 2 * r16 < Rv)
                __stcs(Y + (gc0 + 2 * r16) * ldy + gr,
                       make_double2(cv[r16].x - E[rl * 33 + q], cv[r16].y - E[(64 + rl) * 33 + q]));
            }
          }
        }
        tcp_epi_sync();
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      tcp_epi_sync();
      if (threadIdx.x == 0) tcp_arrive(acce0 + 8 * buf);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_d), "r"(2 * BN) : "memory");
}

template <int BN> constexpr int tcgp_smem() { return TCP_STAGES * (TC_A_STAGE + BN * TC_BK * 4) + TCP_E_BYTES + 256 + 1024; }

// split one complex value into the six 256-strided A'' / B'' segment entries
template <class E>
__device__ __forceinline__ void put_a(E *ar, E *ai, int kk, float vr, float vi) {
  E rh, rl, ih, il;
  split_op(vr, rh, rl);
  split_op(vi, ih, il);
  ar[kk] = rh; ar[256 + kk] = neg_op(ih); ar[512 + kk] = rh; ar[768 + kk] = neg_op(ih); ar[1024 + kk] = rl;
  ar[1280 + kk] = neg_op(il);
  ai[kk] = ih; ai[256 + kk] = rh;  ai[512 + kk] = ih; ai[768 + kk] = rh;  ai[1024 + kk] = il; ai[1280 + kk] = rl;
}

// A'' from a complex matrix: element (m, k) = S[m ld + k] (TRANS: S[k ld + m]),
// zero outside M x K and, with LOWER, unless the element is strictly below the
// diagonal of the source (k < m, or k > m for TRANS: L^T from the lower
// factor).  32 x 32 tiles through shared memory so both the read and the
// write are coalesced; the grid covers exactly Mpad x Kpad.
template <bool TRANS, bool LOWER, class SC, class E>
__global__ void __launch_bounds__(256) k_pack_a(int64_t M, int64_t K, int64_t Kpad, const SC *__restrict__ S,
                                                int64_t ld, E *__restrict__ Ap) {
  __shared__ float2 tile[32][33];
  // LOWER: tiles holding only excluded (zero) elements are not written -- the
  // triangular-sweep GEMMs read the packed factor only in the included part
  if (LOWER && (TRANS ? blockIdx.x < blockIdx.y : blockIdx.x > blockIdx.y)) return;
  const int64_t m0 = (int64_t)blockIdx.y * 32, k0 = (int64_t)blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int i = ty; i < 32; i += 8) {
    if (TRANS) {
      const int64_t k = k0 + i, m = m0 + tx;
      const bool in = m < M && k < K && (!LOWER || k > m);
      const SC v = in ? S[k * ld + m] : SC{};
      tile[tx][i] = make_float2((float)v.x, (float)v.y);
    } else {
      const int64_t m = m0 + i, k = k0 + tx;
      const bool in = m < M && k < K && (!LOWER || k < m);
      const SC v = in ? S[m * ld + k] : SC{};
      tile[i][tx] = make_float2((float)v.x, (float)v.y);
    }
  }
  __syncthreads();
  const int64_t lda = 6 * Kpad;
  for (int i = ty; i < 32; i += 8) {
    const int64_t m = m0 + i, k = k0 + tx;
    const float2 v = tile[i][tx];
    E *ar = Ap + (128 * (m / 64) + m % 64) * lda + (k / 256) * 1536;
    put_a(ar, ar + 64 * lda, (int)(k % 256), v.x, v.y);
  }
}

// B'' from complex128 column-major right-hand sides: row r, complex K index k
// holds X[k + r ldx] (zero for k >= Kv or r >= R).  The grid covers Rpad rows.
template <class E>
__global__ void k_pack_b(int64_t R, int64_t Kv, int64_t Kpad, const double2 *__restrict__ X, int64_t ldx,
                         E *__restrict__ Bp) {
  const int64_t r = blockIdx.y;
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= Kpad) return;
  const double2 v = (r < R && k < Kv) ? X[r * ldx + k] : make_double2(0, 0);
  E rh, rl, ih, il;
  split_op_d(v.x, rh, rl);
  split_op_d(v.y, ih, il);
  E *br = Bp + r * 6 * Kpad + (k / 256) * 1536;
  const int kk = (int)(k % 256);
  br[kk] = rh; br[256 + kk] = ih; br[512 + kk] = rl; br[768 + kk] = il; br[1024 + kk] = rh; br[1280 + kk] = ih;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// 2-D FP32 tensor map over a packed operand: `rows` rows of `ld` floats, boxes
// of 32 floats (one 128-byte swizzle row) x box_rows rows.
void make_map(CUtensorMap *map, float *base, uint64_t rows, uint32_t box_rows, uint64_t ld = TC_K) {
  make_map_bytes(map, base, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, ld, ld * sizeof(float), rows, TC_BK, box_rows);
}
// the same over TF32 (bf false) or BF16 (bf true) elements: boxes of one
// 128-byte row (32 or 64 elements) x box_rows rows
void make_map_op(CUtensorMap *map, void *base, bool bf, uint64_t rows, uint32_t box_rows, uint64_t ld) {
  if (bf)
    make_map_bytes(map, base, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, ld, ld * 2, rows, 64, box_rows);
  else
    make_map_bytes(map, base, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, ld, ld * sizeof(float), rows, TC_BK, box_rows);
}

// factor updates pack their operands into one of TC_UPD_SLOTS buffer pairs,
// one per stream that issues them, so updates of disjoint column ranges run
// concurrently
constexpr int TC_UPD_SLOTS = 3;

struct TcState {
  DevBuf A[TC_UPD_SLOTS], B[TC_UPD_SLOTS], err;
  CUtensorMap mapAK[TC_UPD_SLOTS][4], mapBK[TC_UPD_SLOTS][4];
  int64_t n_key[TC_UPD_SLOTS] = {-1, -1, -1};
  int upd_fmt[TC_UPD_SLOTS] = {-1, -1, -1};  // operand format of the slot's maps (0 TF32, 1 BF16)
  bool attr = false;
  // general GEMMs: packed Z (keyed by the Z version), packed right-hand
  // sides, packed triangular-solve panels
  // Pb: packed right-hand-side blocks of the sweeps, four slots (0: the
  // diagonal-block product, 1-3: the off-diagonal products of successive
  // blocks, read by the lookahead stream too)
  DevBuf Zp, Xp, Pa, Pb[4];
  CUtensorMap mapZ, mapX, mapPaK[4], mapPbK[4][4], mapPbK128[4][4];
  uint64_t zp_version = ~0ull;
  // factor packed once per factorisation for the batched triangular solves:
  // L'' (strict lower), (L^T)'' and the inverses of the 1024-row diagonal
  // blocks of L (forward) and of L^T (backward)
  DevBuf Lp, Ltp, Dfp, Dbp;
  CUtensorMap mapL, mapLt, mapDf, mapDb;
  int64_t lp_n = -1;
  int lp_fmt = -1, pb_fmt[4] = {-1, -1, -1, -1};  // operand formats of the packed factor / of Pb's maps
  int64_t zp_n = -1, xp_key = -1, xp_n = -1, pa_key = -1, pb_key[4] = {-1, -1, -1, -1};
  cudaEvent_t sw_ev[3][4] = {};  // pipelined sweeps: packed / next-block / rest events, ring of 4
  bool gemm_attr = false;
};

int64_t round_up(int64_t v, int64_t m) { return ((v + m - 1) / m) * m; }

std::mutex g_tc_mu;
std::vector<std::pair<dmb_ctx *, TcState *>> g_tc_states;

TcState &tc_state(dmb_ctx *c) {
  std::lock_guard<std::mutex> lk(g_tc_mu);
  for (auto &p : g_tc_states)
    if (p.first == c) return *p.second;
  g_tc_states.push_back({c, new TcState()});
  return *g_tc_states.back().second;
}

void ensure_gemm(dmb_ctx *c, TcState &st) {
  if (!st.err.p) {
    st.err.ensure(16);
    DMB_CUDA(cudaMemsetAsync(st.err.p, 0, 16, c->stream));
  }
  if (!st.gemm_attr) {
    DMB_CUDA(cudaFuncSetAttribute(k_tc_gemm<0, 256, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM));
    DMB_CUDA(cudaFuncSetAttribute(k_tc_gemm<1, 256, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM));
    DMB_CUDA(cudaFuncSetAttribute(k_tc_gemm<1, 128, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM_128));
    DMB_CUDA(cudaFuncSetAttribute(k_tc_gemm<1, 256, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM));
    DMB_CUDA(cudaFuncSetAttribute(k_tc_gemm<1, 128, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM_128));
    DMB_CUDA(cudaFuncSetAttribute(k_tc_gemm_p<256, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  tcgp_smem<256>()));
    DMB_CUDA(cudaFuncSetAttribute(k_tc_gemm_p<256, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  tcgp_smem<256>()));
    st.gemm_attr = true;
  }
}

}  // namespace

namespace dmb {

bool tc_available(dmb_ctx *c) {
  if (!c->use_tensor_cores) return false;
  int major = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, c->device);
  return major == 10 && encode_fn() != nullptr;
}

// Trailing update of the complex64 LDL^T on the tensor cores:
//   F[r][c] -= sum_{k < K} W[r][woff + k] L[c][jcol + k],  r0 <= c < c_hi, c <= r < N
// K <= 1024 (the packed buffers are sized for that).
void tc_ldlt_update_c64(dmb_ctx *c, int64_t N, int64_t r0, int64_t c_hi, int64_t jcol, int K, float2 *F,
                        const float2 *W, int wstride, int woff, int slot) {
  DMB_REQUIRE(K >= 1 && K <= 1024, DMB_ERR_STATE, "tensor-core update width must be 1..1024");
  DMB_REQUIRE(slot >= 0 && slot < TC_UPD_SLOTS, DMB_ERR_STATE, "bad update buffer slot");
  TcState &st = tc_state(c);
  DevBuf &bA = st.A[slot], &bB = st.B[slot];
  const int64_t npadA = ((N + 63) / 64) * 64;
  const int64_t npadB = ((N + TC_BN - 1) / TC_BN) * TC_BN;
  const int64_t Kpad = ((K + 255) / 256) * 256, ld = 6 * Kpad;
  const bool bf = c->pc_bf16();
  if (st.n_key[slot] != N || st.upd_fmt[slot] != (int)bf) {
    bA.ensure(sizeof(float) * 2 * npadA * 6 * 1024);
    bB.ensure(sizeof(float) * npadB * 6 * 1024);
    DMB_CUDA(cudaMemsetAsync(bB.p, 0, sizeof(float) * npadB * 6 * 1024, c->stream));
    for (int i = 0; i < 4; i++) {
      make_map_op(&st.mapAK[slot][i], bA.p, bf, (uint64_t)(2 * npadA), TC_BM, 1536 * (i + 1));
      make_map_op(&st.mapBK[slot][i], bB.p, bf, (uint64_t)npadB, TC_BN, 1536 * (i + 1));
    }
    st.n_key[slot] = N;
    st.upd_fmt[slot] = (int)bf;
  }
  if (!st.err.p) {
    st.err.ensure(16);
    DMB_CUDA(cudaMemsetAsync(st.err.p, 0, 16, c->stream));
  }
  if (!st.attr) {
    DMB_CUDA(cudaFuncSetAttribute(k_tc_syrk<4, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_syrk_smem(4)));
    DMB_CUDA(cudaFuncSetAttribute(k_tc_syrk<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_syrk_smem(2)));
    DMB_CUDA(cudaFuncSetAttribute(k_tc_syrk_p<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, TCP_SMEM));
    DMB_CUDA(cudaFuncSetAttribute(k_tc_syrk<4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_syrk_smem(4)));
    DMB_CUDA(cudaFuncSetAttribute(k_tc_syrk<2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_syrk_smem(2)));
    DMB_CUDA(cudaFuncSetAttribute(k_tc_syrk_p<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, TCP_SMEM));
    st.attr = true;
  }
  const int64_t rest = N - r0, ncols = std::min<int64_t>(c_hi, N) - r0;
  if (rest <= 0 || ncols <= 0) return;
  const int kslot = (int)(Kpad / 256) - 1;
  // A'' rows past `rest` and B'' rows past `ncols` keep stale values: they only
  // feed output rows >= N and columns >= c_hi, which the epilogue skips
  if (bf)
    DMB_LAUNCH(c, k_tc_pack<__nv_bfloat16>, dim3((unsigned)rest, (unsigned)(Kpad / 256)), 256, 0, rest, ncols,
               N, r0, jcol, K, ld, F, W, wstride, woff, bA.as<__nv_bfloat16>(), bB.as<__nv_bfloat16>());
  else
    DMB_LAUNCH(c, k_tc_pack<float>, dim3((unsigned)rest, (unsigned)(Kpad / 256)), 256, 0, rest, ncols,
               N, r0, jcol, K, ld, F, W, wstride, woff, bA.as<float>(), bB.as<float>());
  dim3 grid((unsigned)((rest + 63) / 64), (unsigned)((ncols + TC_BN - 1) / TC_BN));
  const int cpb = (bf ? 8 : 16) * c->precond_tf32_terms;
  // bucket: row tiles (log2) and the K width of the update
  const int64_t tb1 = dmb::tune_bucket((rest + 63) / 64), tb2 = kslot;
  const int cand = dmb::tune_choose(c, dmb::TUNE_TC_SYRK_STAGES, tb1, tb2, 3);
  dmb::TuneMark mk;
  dmb::tune_begin(c, dmb::TUNE_TC_SYRK_STAGES, tb1, tb2, cand, mk);
  if (cand == 2) {
    // persistent: lower tiles only, at most one CTA per SM
    const int nrt = (int)((rest + 63) / 64), nct = (int)((ncols + TC_BN - 1) / TC_BN);
    int64_t ntiles = 0;
    for (int ct = 0; ct < nct; ct++) ntiles += std::max<int64_t>(0, nrt - 4 * ct);
    const unsigned G = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ntiles, c->sm_count));
    if (ntiles > 0) {
      if (bf)
        DMB_LAUNCH(c, k_tc_syrk_p<true>, G, 192, TCP_SMEM, st.mapAK[slot][kslot], st.mapBK[slot][kslot], F, N, r0,
                   std::min<int64_t>(c_hi, N), (int)(Kpad / 256) * cpb, cpb, nrt, nct, ntiles,
                   st.err.as<unsigned>());
      else
        DMB_LAUNCH(c, k_tc_syrk_p<false>, G, 192, TCP_SMEM, st.mapAK[slot][kslot], st.mapBK[slot][kslot], F, N,
                   r0, std::min<int64_t>(c_hi, N), (int)(Kpad / 256) * cpb, cpb, nrt, nct, ntiles,
                   st.err.as<unsigned>());
    }
  } else {
#define SYRK_LAUNCH(STG, BFV)                                                                                     \
  DMB_LAUNCH(c, (k_tc_syrk<STG, BFV>), grid, 128, tc_syrk_smem(STG), st.mapAK[slot][kslot], st.mapBK[slot][kslot], \
             F, N, r0, rest, std::min<int64_t>(c_hi, N), (int)(Kpad / 256) * cpb, cpb, st.err.as<unsigned>())
    if (cand == 0) {
      if (bf) SYRK_LAUNCH(4, true);
      else SYRK_LAUNCH(4, false);
    } else {
      if (bf) SYRK_LAUNCH(2, true);
      else SYRK_LAUNCH(2, false);
    }
#undef SYRK_LAUNCH
  }
  dmb::tune_end(c, mk);
}

unsigned tc_error_word(dmb_ctx *c) {
  TcState &st = tc_state(c);
  if (!st.err.p) return 0;
  unsigned e = 0;
  DMB_CUDA(cudaMemcpyAsync(&e, st.err.p, 4, cudaMemcpyDeviceToHost, c->stream));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  return e;
}

// Packed Z (re-packed whenever Z changes), Y = Z X for R right-hand sides
// (X, Y complex128 column-major N x R) on the tensor cores.
void tc_zx(dmb_ctx *c, const double2 *X, double2 *Y, int64_t R) {
  DMB_REQUIRE(c->z_prec == DMB_PREC_MIXED, DMB_ERR_STATE, "tensor-core Z X needs the complex64 matrix");
  TcState &st = tc_state(c);
  ensure_gemm(c, st);
  const int64_t N = c->n, Kpad = round_up(N, 256), Mpad = round_up(N, 64), Rpad = round_up(R, TC_BN);
  const int64_t ld = 6 * Kpad;
  if (st.zp_version != c->z_version || st.zp_n != N) {
    st.Zp.ensure(sizeof(float) * 2 * Mpad * ld);
    dim3 g((unsigned)(Kpad / 32), (unsigned)(Mpad / 32));
    DMB_LAUNCH(c, (k_pack_a<false, false, float2, float>), g, 256, 0, N, N, Kpad, c->d_Z.as<float2>(), N,
               st.Zp.as<float>());
    make_map(&st.mapZ, st.Zp.as<float>(), (uint64_t)(2 * Mpad), TC_BM, (uint64_t)ld);
    st.zp_version = c->z_version;
    st.zp_n = N;
  }
  st.Xp.ensure(sizeof(float) * Rpad * ld);
  if (st.xp_key != Rpad || st.xp_n != N) {
    make_map(&st.mapX, st.Xp.as<float>(), (uint64_t)Rpad, TC_BN, (uint64_t)ld);
    st.xp_key = Rpad;
    st.xp_n = N;
  }
  DMB_LAUNCH(c, k_pack_b<float>, dim3((unsigned)(Kpad / 256), (unsigned)Rpad), 256, 0, R, N, Kpad, X, N,
             st.Xp.as<float>());
  dim3 grid((unsigned)(Rpad / TC_BN), (unsigned)(Mpad / 64));
  kt_begin(c);
  DMB_LAUNCH(c, (k_tc_gemm<0, 256, false>), grid, 128, TC_SMEM, st.mapZ, st.mapX, 0, 0, (int)(ld / TC_BK), 48, N, R, Y, N, 0, 0,
             st.err.as<unsigned>());
  kt_end(c, 8.0 * (double)N * (double)N * (double)R);
}

// One update of the batched triangular solves with the complex64 factor F
// (L strictly lower, row-major N x N), rows [r_lo, r_hi), K = [k_lo, k_lo + w):
//   forward:  X[r_lo : r_hi] -= L[r_lo : r_hi, k_lo : k_lo + w]   X[k_lo : k_lo + w]
//   backward: X[r_lo : r_hi] -= L[k_lo : k_lo + w, r_lo : r_hi]^T X[k_lo : k_lo + w]
// w <= 1024.  The packed panels live in buffers sized for w = 1024; one tensor
// map per (buffer, K width) is kept.
void tc_trsm_update(dmb_ctx *c, const float2 *F, int64_t N, int64_t r_lo, int64_t r_hi, int64_t k_lo, int width,
                    bool backward, double2 *X, int64_t R) {
  DMB_REQUIRE(width >= 1 && width <= 1024, DMB_ERR_STATE, "panel width must be 1..1024");
  TcState &st = tc_state(c);
  ensure_gemm(c, st);
  const int64_t M = r_hi - r_lo;
  if (M <= 0) return;
  const int64_t Npad = round_up(N, 64), Mpad = round_up(M, 64), Rpad = round_up(R, TC_BN);
  const int64_t Kpad = round_up(width, 256), ld = 6 * Kpad;
  const int kslot = (int)(Kpad / 256) - 1;  // 0..3
  if (st.pa_key != Npad) {
    st.Pa.ensure(sizeof(float) * 2 * Npad * 6 * 1024);
    for (int i = 0; i < 4; i++) make_map(&st.mapPaK[i], st.Pa.as<float>(), (uint64_t)(2 * Npad), TC_BM, 1536 * (i + 1));
    st.pa_key = Npad;
  }
  if (st.pb_key[0] != Rpad || st.pb_fmt[0] != 0) {
    st.Pb[0].ensure(sizeof(float) * Rpad * 6 * 1024);
    for (int i = 0; i < 4; i++) {
      make_map(&st.mapPbK[0][i], st.Pb[0].as<float>(), (uint64_t)Rpad, TC_BN, 1536 * (i + 1));
      make_map(&st.mapPbK128[0][i], st.Pb[0].as<float>(), (uint64_t)Rpad, 128, 1536 * (i + 1));
    }
    st.pb_key[0] = Rpad;
    st.pb_fmt[0] = 0;
  }
  dim3 ga((unsigned)(Kpad / 32), (unsigned)(Mpad / 32));
  if (backward)
    DMB_LAUNCH(c, (k_pack_a<true, false, float2, float>), ga, 256, 0, M, (int64_t)width, Kpad, F + k_lo * N + r_lo,
               N, st.Pa.as<float>());
  else
    DMB_LAUNCH(c, (k_pack_a<false, false, float2, float>), ga, 256, 0, M, (int64_t)width, Kpad, F + r_lo * N + k_lo,
               N, st.Pa.as<float>());
  DMB_LAUNCH(c, k_pack_b<float>, dim3((unsigned)(Kpad / 256), (unsigned)Rpad), 256, 0, R, (int64_t)width, Kpad,
             X + k_lo, N, st.Pb[0].as<float>());
  dim3 grid((unsigned)(Rpad / TC_BN), (unsigned)(Mpad / 64));
  kt_begin(c);
  DMB_LAUNCH(c, (k_tc_gemm<1, 256, false>), grid, 128, TC_SMEM, st.mapPaK[kslot], st.mapPbK[0][kslot], 0, 0, (int)(ld / TC_BK), 48, M, R,
             X + r_lo, N, 1, 0, st.err.as<unsigned>());
  kt_end(c, 8.0 * (double)M * (double)width * (double)R);
}

// ---- batched triangular solves with the factor packed once ---------------
constexpr int TB = 1024;  // outer block rows

// L'' and (L^T)'' of the complex64 factor (strict lower part of F)
void tc_trsm_pack_factor(dmb_ctx *c, const float2 *F, int64_t N) {
  TcState &st = tc_state(c);
  ensure_gemm(c, st);
  const int64_t Mpad = round_up(N, 64), Kpad = round_up(N, 256), ld = 6 * Kpad;
  const int64_t nout = (N + TB - 1) / TB;
  const bool bf = c->pc_bf16();
  if (st.lp_n != N || st.lp_fmt != (int)bf) {
    st.Lp.ensure(sizeof(float) * 2 * Mpad * ld);
    st.Ltp.ensure(sizeof(float) * 2 * Mpad * ld);
    st.Dfp.ensure(sizeof(float) * 2 * TB * nout * 6 * TB);
    st.Dbp.ensure(sizeof(float) * 2 * TB * nout * 6 * TB);
    make_map_op(&st.mapL, st.Lp.p, bf, (uint64_t)(2 * Mpad), TC_BM, (uint64_t)ld);
    make_map_op(&st.mapLt, st.Ltp.p, bf, (uint64_t)(2 * Mpad), TC_BM, (uint64_t)ld);
    make_map_op(&st.mapDf, st.Dfp.p, bf, (uint64_t)(2 * TB * nout), TC_BM, 6 * TB);
    make_map_op(&st.mapDb, st.Dbp.p, bf, (uint64_t)(2 * TB * nout), TC_BM, 6 * TB);
    // diagonal-block buffers: rows of a short last block stay zero
    DMB_CUDA(cudaMemsetAsync(st.Dfp.p, 0, st.Dfp.bytes, c->stream));
    DMB_CUDA(cudaMemsetAsync(st.Dbp.p, 0, st.Dbp.bytes, c->stream));
    st.lp_n = N;
    st.lp_fmt = (int)bf;
  }
  dim3 g((unsigned)(Kpad / 32), (unsigned)(Mpad / 32));
  if (bf) {
    DMB_LAUNCH(c, (k_pack_a<false, true, float2, __nv_bfloat16>), g, 256, 0, N, N, Kpad, F, N,
               st.Lp.as<__nv_bfloat16>());
    DMB_LAUNCH(c, (k_pack_a<true, true, float2, __nv_bfloat16>), g, 256, 0, N, N, Kpad, F, N,
               st.Ltp.as<__nv_bfloat16>());
  } else {
    DMB_LAUNCH(c, (k_pack_a<false, true, float2, float>), g, 256, 0, N, N, Kpad, F, N, st.Lp.as<float>());
    DMB_LAUNCH(c, (k_pack_a<true, true, float2, float>), g, 256, 0, N, N, Kpad, F, N, st.Ltp.as<float>());
  }
}

// inverse of diagonal block o (ow x ow, column-major in Xb with leading
// dimension ld) -> forward operand, its transpose -> backward operand
void tc_trsm_pack_diag(dmb_ctx *c, int64_t o, const double2 *Xb, int64_t ld, int ow) {
  TcState &st = tc_state(c);
  dim3 g(TB / 32, TB / 32);
  // in the format of the packed factor (tc_trsm_pack_factor ran first)
  if (st.lp_fmt == 1) {
    __nv_bfloat16 *df = st.Dfp.as<__nv_bfloat16>() + o * 2 * TB * 6 * TB;
    __nv_bfloat16 *db = st.Dbp.as<__nv_bfloat16>() + o * 2 * TB * 6 * TB;
    DMB_LAUNCH(c, (k_pack_a<true, false, double2, __nv_bfloat16>), g, 256, 0, (int64_t)ow, (int64_t)ow, (int64_t)TB,
               Xb, ld, df);
    DMB_LAUNCH(c, (k_pack_a<false, false, double2, __nv_bfloat16>), g, 256, 0, (int64_t)ow, (int64_t)ow,
               (int64_t)TB, Xb, ld, db);
    return;
  }
  float *df = st.Dfp.as<float>() + o * 2 * TB * 6 * TB;
  float *db = st.Dbp.as<float>() + o * 2 * TB * 6 * TB;
  // forward: A(m, k) = Linv[m][k] = Xb[m + k ld]
  DMB_LAUNCH(c, (k_pack_a<true, false, double2, float>), g, 256, 0, (int64_t)ow, (int64_t)ow, (int64_t)TB, Xb, ld,
             df);
  // backward: A(m, k) = Linv[k][m] = Xb[k + m ld]
  DMB_LAUNCH(c, (k_pack_a<false, false, double2, float>), g, 256, 0, (int64_t)ow, (int64_t)ow, (int64_t)TB, Xb, ld,
             db);
}

// B'' of the sweeps: X[k0 : k0 + w] (R columns) packed into slot `slot`
void pack_b_slot(dmb_ctx *c, TcState &st, int slot, int w, const double2 *Xk, int64_t N, int64_t R) {
  const int64_t Kpad = round_up(w, 256), Rpad = round_up(R, TC_BN);
  const bool bf = st.lp_fmt == 1;  // operands in the format of the packed factor
  if (st.pb_key[slot] != Rpad || st.pb_fmt[slot] != (int)bf) {
    st.Pb[slot].ensure(sizeof(float) * Rpad * 6 * 1024);
    for (int i = 0; i < 4; i++) {
      make_map_op(&st.mapPbK[slot][i], st.Pb[slot].p, bf, (uint64_t)Rpad, TC_BN, 1536 * (i + 1));
      make_map_op(&st.mapPbK128[slot][i], st.Pb[slot].p, bf, (uint64_t)Rpad, 128, 1536 * (i + 1));
    }
    st.pb_key[slot] = Rpad;
    st.pb_fmt[slot] = (int)bf;
  }
  if (bf)
    DMB_LAUNCH(c, k_pack_b<__nv_bfloat16>, dim3((unsigned)(Kpad / 256), (unsigned)Rpad), 256, 0, R, (int64_t)w,
               Kpad, Xk, N, st.Pb[slot].as<__nv_bfloat16>());
  else
    DMB_LAUNCH(c, k_pack_b<float>, dim3((unsigned)(Kpad / 256), (unsigned)Rpad), 256, 0, R, (int64_t)w, Kpad, Xk,
               N, st.Pb[slot].as<float>());
}

// Y (op)= A_packed[rows a_row0.., K from a_kx0] * B'' of slot `slot` (K = w)
void gemm_packed(dmb_ctx *c, TcState &st, int slot, const CUtensorMap &mapA, int a_row0, int a_kx0, int64_t M,
                 int w, double2 *Y, int64_t N, int64_t R, int mode, int tri) {
  if (M <= 0) return;
  const int64_t Kpad = round_up(w, 256), Mpad = round_up(M, 64), Rpad = round_up(R, TC_BN);
  const int kslot = (int)(Kpad / 256) - 1;
  const bool bf = st.lp_fmt == 1;
  // launch shape from the autotuner, per (row tiles, columns, triangular
  // kind): one CTA per 64 x 256 or 64 x 128 complex tile (128 doubles the
  // CTAs of launches with few row tiles), or the persistent 256-wide form (one
  // CTA per SM, a tile's epilogue overlapping the next tile's main loop; it
  // pays only with several tiles per CTA); all three give the same bits
  const int64_t tb1 = dmb::tune_bucket(Mpad / 64), tb2 = (Rpad / 128) * 4 + tri;
  const int cand = dmb::tune_choose(c, dmb::TUNE_TC_GEMM_BN, tb1, tb2, 3);
  const int cpb = (bf ? 8 : 16) * c->precond_tf32_terms;
  const int nchunks = (int)(Kpad / 256) * cpb;
  dmb::TuneMark mk;
  dmb::tune_begin(c, dmb::TUNE_TC_GEMM_BN, tb1, tb2, cand, mk);
  kt_begin(c);
  if (cand < 2) {
#define GEMM_LAUNCH(BNV, BFV, MAPB, SMEMV)                                                                       \
  DMB_LAUNCH(c, (k_tc_gemm<1, BNV, BFV>), dim3((unsigned)(Rpad / BNV), (unsigned)(Mpad / 64)), 128, SMEMV, mapA, \
             MAPB[kslot], a_row0, a_kx0, nchunks, cpb, M, R, Y, N, mode, tri, st.err.as<unsigned>())
    if (cand == 1) {
      if (bf) GEMM_LAUNCH(128, true, st.mapPbK128[slot], TC_SMEM_128);
      else GEMM_LAUNCH(128, false, st.mapPbK128[slot], TC_SMEM_128);
    } else {
      if (bf) GEMM_LAUNCH(256, true, st.mapPbK[slot], TC_SMEM);
      else GEMM_LAUNCH(256, false, st.mapPbK[slot], TC_SMEM);
    }
#undef GEMM_LAUNCH
  } else {
    // tiles: Mpad / 64 row tiles x ceil(R / 256) column tiles, column fastest
    const int ntc = (int)((R + 255) / 256);
    const int64_t ntiles = (Mpad / 64) * ntc;
    const unsigned G = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ntiles, c->sm_count));
    if (bf)
      DMB_LAUNCH(c, (k_tc_gemm_p<256, true>), dim3(G), 192, tcgp_smem<256>(), mapA, st.mapPbK[slot][kslot], a_row0, a_kx0,
                 nchunks, cpb, M, R, Y, N, mode, tri, ntc, ntiles, st.err.as<unsigned>());
    else
      DMB_LAUNCH(c, (k_tc_gemm_p<256, false>), dim3(G), 192, tcgp_smem<256>(), mapA, st.mapPbK[slot][kslot], a_row0,
                 a_kx0, nchunks, cpb, M, R, Y, N, mode, tri, ntc, ntiles, st.err.as<unsigned>());
  }
  // a triangular A does half the MACs
  kt_end(c, (tri ? 4.0 : 8.0) * (double)M * (double)w * (double)R);
  dmb::tune_end(c, mk);
}


// Y (op)= A_packed[rows a_row0.., K from a_kx0] * X[k0 : k0 + w], B packed here
void gemm_prepacked(dmb_ctx *c, TcState &st, const CUtensorMap &mapA, int a_row0, int a_kx0, int64_t M, int w,
                    const double2 *Xk, double2 *Y, int64_t N, int64_t R, int mode, int tri) {
  if (M <= 0) return;
  pack_b_slot(c, st, 0, w, Xk, N, R);
  gemm_packed(c, st, 0, mapA, a_row0, a_kx0, M, w, Y, N, R, mode, tri);
}

// one sweep of the batched solve with the packed factor:
//   forward  (L y = x):   per block o: X_o = Linv_o X_o; X[o1:] -= L[o1:, o] X_o
//   backward (L^T x = z): per block o, last first: X_o = Linv_o^T X_o;
//                         X[:o0] -= L[o, :o0]^T X_o
void tc_trsm_sweep(dmb_ctx *c, int64_t N, double2 *X, int64_t R, bool backward) {
  TcState &st = tc_state(c);
  DMB_REQUIRE(st.lp_n == N, DMB_ERR_STATE, "factor not packed for the batched solves");
  const int64_t nout = (N + TB - 1) / TB;
  // Pipelined over two streams.  Main stream, per block o: the diagonal-block
  // product (X_o = Linv_o X_o, B'' in slot 0), X_o packed into slot 1 +
  // o mod 3, then the update of the block the sweep meets next (the critical
  // one).  Lookahead stream: the update of the block after that, then of all
  // remaining rows.  Each row block is updated by one stream at a time:
  // before block o's diagonal product the main stream waits for the
  // lookahead update of block o made by block o - 2 (which follows every
  // earlier lookahead update), and before its critical update of block o + 1
  // for the one made by block o - 1.  A packed slot is reused three blocks
  // later, after the main stream has waited for a later lookahead event.
  if (!c->stream2) {
    int least = 0, greatest = 0;
    DMB_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    const int mid = greatest < least ? greatest + 1 : least;
    DMB_CUDA(cudaStreamCreateWithPriority(&c->stream2, cudaStreamNonBlocking, mid));
  }
  for (auto &row : st.sw_ev)
    for (auto &e : row)
      if (!e) DMB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaEvent_t *ev_pack = st.sw_ev[0], *ev_next = st.sw_ev[1], *ev_rest = st.sw_ev[2];
  // rows of the block the sweep meets s blocks after block o (-1 for none)
  auto block_rows = [&](int64_t o, int64_t s, int64_t &r0, int64_t &r1) {
    const int64_t q = backward ? o - s : o + s;
    if (q < 0 || q >= nout) return false;
    r0 = q * TB;
    r1 = std::min<int64_t>(N, r0 + TB);
    return true;
  };
  for (int64_t s = 0; s < nout; s++) {
    const int64_t o = backward ? nout - 1 - s : s;
    const int64_t o0 = o * TB, o1 = std::min<int64_t>(N, o0 + TB);
    const int ow = (int)(o1 - o0);
    const int slot = 1 + (int)(s % 3);
    if (s >= 2) DMB_CUDA(cudaStreamWaitEvent(c->stream, ev_next[(s - 2) % 4], 0));
    gemm_prepacked(c, st, backward ? st.mapDb : st.mapDf, (int)(2 * TB * o), 0, ow, ow, X + o0, X + o0, N, R, 0,
                   backward ? 2 : 1);
    pack_b_slot(c, st, slot, ow, X + o0, N, R);
    DMB_CUDA(cudaEventRecord(ev_pack[s % 4], c->stream));
    // the off-diagonal product on rows [ra, rb): backward reads rows of the
    // packed L^T'' (K from o0), forward rows of L''
    auto update = [&](int64_t ra, int64_t rb) {
      if (rb <= ra) return;
      if (backward)
        gemm_packed(c, st, slot, st.mapLt, (int)(2 * ra), (int)(6 * o0), rb - ra, ow, X + ra, N, R, 1, 0);
      else
        gemm_packed(c, st, slot, st.mapL, (int)(2 * ra), (int)(6 * o0), rb - ra, ow, X + ra, N, R, 1, 0);
    };
    int64_t c0, c1;
    if (block_rows(o, 1, c0, c1)) {
      if (s >= 1) DMB_CUDA(cudaStreamWaitEvent(c->stream, ev_next[(s - 1) % 4], 0));
      update(c0, c1);
    }
    {
      StreamSwap sw(c, c->stream2);
      DMB_CUDA(cudaStreamWaitEvent(c->stream, ev_pack[s % 4], 0));
      int64_t n0, n1;
      if (block_rows(o, 2, n0, n1)) update(n0, n1);
      DMB_CUDA(cudaEventRecord(ev_next[s % 4], c->stream));
      // the rest: rows beyond the block after next
      if (backward) {
        int64_t e0, e1;
        if (block_rows(o, 3, e0, e1)) update(0, e1);
      } else {
        int64_t e0, e1;
        if (block_rows(o, 3, e0, e1)) update(e0, N);
      }
      DMB_CUDA(cudaEventRecord(ev_rest[s % 4], c->stream));
    }
  }
  // the sweep ends when the lookahead stream is done
  DMB_CUDA(cudaStreamWaitEvent(c->stream, ev_rest[(nout - 1) % 4], 0));
}

// drop the context's packed operands (called when the context is destroyed)
void tc_release(dmb_ctx *c) {
  std::lock_guard<std::mutex> lk(g_tc_mu);
  for (size_t i = 0; i < g_tc_states.size(); i++) {
    if (g_tc_states[i].first != c) continue;
    TcState *st = g_tc_states[i].second;
    for (DevBuf *b : {&st->err, &st->Zp, &st->Xp, &st->Pa, &st->Pb[0], &st->Pb[1], &st->Pb[2], &st->Pb[3],
                      &st->Lp, &st->Ltp, &st->Dfp, &st->Dbp})
      b->release();
    for (auto &row : st->sw_ev)
      for (auto &e : row)
        if (e) cudaEventDestroy(e);
    for (int slot = 0; slot < TC_UPD_SLOTS; slot++) {
      st->A[slot].release();
      st->B[slot].release();
    }
    delete st;
    g_tc_states.erase(g_tc_states.begin() + i);
    return;
  }
}

}  // namespace dmb
