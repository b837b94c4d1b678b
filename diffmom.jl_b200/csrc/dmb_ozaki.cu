// dmb_ozaki.cu -- FP64-accurate Y = Z X for a complex64 Z and complex128 X on
// the INT8 tensor cores (tcgen05.mma.kind::i8, exact int32 accumulation):
// the refinement and true residuals of the batched solves.
//
// Method (error-free splitting, Ozaki, Ogita, Oishi & Rump, "Error-free
// transformations of matrix multiplication by using fast routines of matrix
// multiplication and its applications", Numer. Algorithms 59, 2012, here with
// fixed-point int8 slices):
//   * complex as one real product: row m of Z gives a real row [Zr, -Zi] and an
//     imaginary row [Zi, Zr] against the column [Xr; Xi] (K = 2N);
//   * each complex row m is scaled by sigma_m = 2^e (the smallest power of two
//     above max_k max(|Zr|, |Zi|)), each column r of X by tau_r likewise, and
//     the scaled values in (-1, 1) are cut into OZ_S slices of OZ_BETA = 7
//     bits, v = sum_p a_p 2^(-7(p+1)) with integer a_p in [-127, 127] (exact in
//     double arithmetic);
//   * slice products a_p . b_q are exact in int32 (127^2 x 2N < 2^31 per pair);
//     pairs with p + q <= OZ_LMAX (0-based) are kept, summed in TMEM per level
//     (as many pairs per drain as int32 allows) and drained into FP64 with the
//     exact power-of-two weights sigma_m tau_r 2^(-7(L+2)).
// With OZ_S = 6 and all levels up to OZ_LMAX = 6 (26 int8 products) the
// product is ~7e-13 relative (normwise) on EFIE rows; the Krylov products of
// GMRES keep levels <= 5 (21 products, ~4e-11), the true residuals all levels.
//
// Kernel k_oz_gemm: a persistent grid (one CTA per SM) over 64 x 256 complex
// output tiles -- whole tiles in data-parallel waves, the tail tiles split
// stream-K and summed by k_oz_fixup -- 6 warps per CTA:
//   warp 4 / lane 0   TMA producer over (pair, K chunk) into a 4-stage ring of
//                     128-byte-swizzled int8 stages (A 128 x 128 B, B 256 x 128 B);
//   warp 5 / lane 0   tcgen05.mma.kind::i8 (M 128, N 256, K 32) into two
//                     256-column s32 TMEM accumulators used in turn (one
//                     level accumulates while the other drains), one commit
//                     per drain;
//   warps 0-3         drain each level: tcgen05.ld, scale, FP64 store / add.
// Every wait is bounded (error bit, abort flag, TMEM freed); no multicast.
#include <algorithm>
#include <vector>
#include <cmath>

#include "dmb_device.cuh"
#include "dmb_internal.h"
#include "dmb_tcgen05.cuh"

namespace {

using namespace dmb_tc;

constexpr int OZ_BETA = 7;
constexpr int OZ_S = 6;
constexpr int OZ_LMAX = 6;
constexpr int OZ_MAXP = OZ_S * OZ_S;
constexpr int OZ_BM = 128, OZ_BN = 256, OZ_BK = 128;  // BK in bytes (= int8 K elements)
constexpr int OZ_STAGES = 4;
constexpr int OZ_A_STAGE = OZ_BM * OZ_BK, OZ_B_STAGE = OZ_BN * OZ_BK;
constexpr int OZ_E_BYTES = OZ_BM * 33 * 4;
constexpr int OZ_SMEM = OZ_STAGES * (OZ_A_STAGE + OZ_B_STAGE) + OZ_E_BYTES + 256 /*barriers*/ + 1024 /*align*/;
// D s32, A/B signed int8, K-major, N = 256, M = 128
constexpr uint32_t OZ_IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(OZ_BN >> 3) << 17) |
                              ((uint32_t)(OZ_BM >> 4) << 24);

struct OzSched {
  int n;
  int arow[OZ_MAXP];      // first A'' row of the pair's Z slice
  int brow[OZ_MAXP];      // first B'' row of the pair's X slice
  int close[OZ_MAXP];     // 1: the TMEM sum is drained after this pair
  double lscale[OZ_MAXP]; // weight of the pair's level: 2^(-7 (L + 2))
};

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(OZ_IDESC), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

// Persistent grid of G CTAs over ntiles output tiles (column tile fastest).
// The first nfull = ntiles / G waves are data-parallel: CTA b computes tiles
// b, b + G, ... whole, so the CTAs running together share the Z slices of a
// row of tiles in L2.  The remaining tail tiles are split stream-K: their
// units (tile, slice pair) are cut into G equal ranges; a range's segment that
// covers a whole tile writes Y, the (at most two) partial segments of a range
// go to the CTA's workspace slots, and k_oz_fixup sums each tile's partials in
// CTA order.  Every role walks the same sequence of segments and of drain
// groups (a level's pairs, cut at sc.close and at the segment end).
struct OzSeg {
  int64_t t;
  int p0, p1, slot;  // slot -1: whole tile into Y
};
struct OzIter {
  int64_t wave, nfull, b, G, u, u_end;
  int n, slot;
};
__device__ __forceinline__ void oz_iter_init(OzIter &it, int64_t ntiles, int n) {
  it.G = gridDim.x;
  it.b = blockIdx.x;
  it.n = n;
  it.wave = 0;
  it.nfull = ntiles / it.G;
  const int64_t F = it.nfull * it.G, Wt = (ntiles - F) * n;
  it.u = F * n + Wt * it.b / it.G;
  it.u_end = F * n + Wt * (it.b + 1) / it.G;
  it.slot = 0;
}
__device__ __forceinline__ bool oz_next_seg(OzIter &it, OzSeg &sg) {
  if (it.wave < it.nfull) {
    sg.t = it.wave * it.G + it.b;
    sg.p0 = 0;
    sg.p1 = it.n;
    sg.slot = -1;
    it.wave++;
    return true;
  }
  if (it.u >= it.u_end) return false;
  sg.t = it.u / it.n;
  sg.p0 = (int)(it.u - sg.t * it.n);
  sg.p1 = (int)min((int64_t)it.n, it.u_end - sg.t * it.n);
  it.u = sg.t * it.n + sg.p1;
  sg.slot = (sg.p0 == 0 && sg.p1 == it.n) ? -1 : it.slot++;
  return true;
}
constexpr int OZ_TILE_ELEMS = 64 * OZ_BN;  // complex outputs per tile (workspace slot size)

__global__ void __launch_bounds__(192, 1) k_oz_gemm(const __grid_constant__ CUtensorMap tmA,
                                                    const __grid_constant__ CUtensorMap tmB,
                                                    const __grid_constant__ OzSched sc, int kchunks, int64_t M,
                                                    int64_t Rv, double2 *__restrict__ Y, double2 *__restrict__ P,
                                                    int64_t ldy, int ncol, int64_t ntiles,
                                                    const double *__restrict__ rs, const double *__restrict__ cs,
                                                    unsigned *err) {

  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char *gbase = smem_raw + (base - raw);
  const uint32_t sA = base;
  const uint32_t sB = base + OZ_STAGES * OZ_A_STAGE;
  int *E = reinterpret_cast<int *>(gbase + OZ_STAGES * (OZ_A_STAGE + OZ_B_STAGE));
  const uint32_t sBar = sB + OZ_STAGES * OZ_B_STAGE + OZ_E_BYTES;
  uint64_t *bar_ptr = reinterpret_cast<uint64_t *>(gbase + (sBar - base));
  volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(bar_ptr + 16);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(bar_ptr + 17);
  volatile int *epi_ok = reinterpret_cast<volatile int *>(bar_ptr + 18);
  // accf[b] / acce[b]: TMEM accumulator b (of two) full / drained
  const uint32_t full0 = sBar, empty0 = sBar + 8 * OZ_STAGES, accf0 = sBar + 16 * OZ_STAGES, acce0 = accf0 + 16;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < OZ_STAGES; s++) {
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
                 "r"(2 * OZ_BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem_d = *tmem_slot;

  if (warp == 4) {
    if (lane == 0) {
      long long t = 0;
      OzIter it;
      oz_iter_init(it, ntiles, sc.n);
      OzSeg sg;
      bool go = true;
      while (go && oz_next_seg(it, sg)) {
        const int row2 = (int)(2 * 64 * (sg.t / ncol)), colb = (int)(OZ_BN * (sg.t % ncol));
        for (int i = sg.p0; i < sg.p1 && go; i++) {
          for (int kc = 0; kc < kchunks; kc++, t++) {
            const int s = (int)(t % OZ_STAGES);
            if (*abort_flag ||
                (t >= OZ_STAGES && !mbar_wait(empty0 + 8 * s, (uint32_t)((t / OZ_STAGES) - 1) & 1u, err, abort_flag))) {
              go = false;
              break;
            }
            mbar_expect_tx(full0 + 8 * s, OZ_A_STAGE + OZ_B_STAGE);
            tma_load_2d(sA + s * OZ_A_STAGE, &tmA, kc * OZ_BK, sc.arow[i] + row2, full0 + 8 * s);
            tma_load_2d(sB + s * OZ_B_STAGE, &tmB, kc * OZ_BK, sc.brow[i] + colb, full0 + 8 * s);
          }
        }
      }
    }
  } else if (warp == 5) {
    if (lane == 0) {
      long long t = 0;
      int g = 0;
      bool ok = true;
      OzIter it;
      oz_iter_init(it, ntiles, sc.n);
      OzSeg sg;
      while (ok && oz_next_seg(it, sg)) {
        bool first = true;
        for (int i = sg.p0; i < sg.p1 && ok; i++) {
          // group g accumulates in buffer g & 1, free once group g - 2 drained
          if (first && g >= 2 &&
              !mbar_wait(acce0 + 8 * (g & 1), (uint32_t)((g >> 1) - 1) & 1u, err, abort_flag)) {
            ok = false;
            break;
          }
          const uint32_t tmem_acc = tmem_d + (uint32_t)((g & 1) * OZ_BN);
          for (int kc = 0; kc < kchunks; kc++, t++) {
            const int s = (int)(t % OZ_STAGES);
            if (!mbar_wait(full0 + 8 * s, (uint32_t)(t / OZ_STAGES) & 1u, err, abort_flag)) {
              ok = false;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int k = 0; k < OZ_BK / 32; k++) {
              const uint64_t ad = sw128_desc(sA + s * OZ_A_STAGE + k * 32);
              const uint64_t bd = sw128_desc(sB + s * OZ_B_STAGE + k * 32);
              umma_i8(tmem_acc, ad, bd, (first && kc == 0 && k == 0) ? 0u : 1u);
            }
            umma_commit(empty0 + 8 * s);
          }
          first = false;
          if (ok && (sc.close[i] || i + 1 == sg.p1)) {
            umma_commit(accf0 + 8 * (g & 1));
            g++;
            first = true;
          }
        }
      }
    }
  } else {
    // drain warps 0-3 (warp w reads TMEM lanes 32w..32w+31)
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    const int rl = threadIdx.x & 63, qh = threadIdx.x >> 6;
    int g = 0;
    bool alive = true;
    OzIter it;
    oz_iter_init(it, ntiles, sc.n);
    OzSeg sg;
    while (alive && oz_next_seg(it, sg)) {
    const int64_t row0 = 64 * (sg.t / ncol), col0 = (int64_t)OZ_BN * (sg.t % ncol);
    // target of this segment: its tile of Y, or a workspace slot (64 x 256,
    // column-major with leading dimension 64)
    double2 *Yt = sg.slot < 0 ? Y + col0 * ldy + row0 : P + ((int64_t)blockIdx.x * 2 + sg.slot) * OZ_TILE_ELEMS;
    const int64_t ldt = sg.slot < 0 ? ldy : 64;
    const int64_t gr = row0 + rl;
    const double rsc = gr < M ? rs[gr] : 0.0;
    for (int i = sg.p0, gi = 0; i < sg.p1; gi++) {
      // the group: pairs i .. j, cut at the level's drain point or the segment end
      int j = i;
      while (!sc.close[j] && j + 1 < sg.p1) j++;
      const double gsc = sc.lscale[i];
      i = j + 1;
      const bool got = mbar_wait(accf0 + 8 * (g & 1), (uint32_t)(g >> 1) & 1u, err, abort_flag);
      const uint32_t tmem_acc = tmem_d + (uint32_t)((g & 1) * OZ_BN);
      if (threadIdx.x == 0) *epi_ok = 1;
      epi_sync();
      if (!got) *epi_ok = 0;
      epi_sync();
      if (!*epi_ok) {
        alive = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int cc = 0; cc < OZ_BN / 32; cc++) {
        if (col0 + cc * 32 >= Rv) break;  // uniform over the drain warps
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
        for (int q = 0; q < 32; q++) E[row * 33 + q] = (int)v[q];
        epi_sync();
        if (gr < M) {
          const int64_t gc0 = col0 + cc * 32 + qh;
          double2 old[16];
          if (gi > 0) {
#pragma unroll
            for (int x = 0; x < 16; x++)
              old[x] = (gc0 + 2 * x < Rv) ? Yt[(gc0 + 2 * x - col0) * ldt + rl] : make_double2(0, 0);
          } else {
#pragma unroll
            for (int x = 0; x < 16; x++) old[x] = make_double2(0, 0);
          }
#pragma unroll
          for (int x = 0; x < 16; x++) {
            const int q = qh + 2 * x;
            const int64_t gc = gc0 + 2 * x;
            if (gc < Rv) {
              const double w = rsc * cs[gc] * gsc;
              Yt[(gc - col0) * ldt + rl] = make_double2(fma((double)E[rl * 33 + q], w, old[x].x),
                                                        fma((double)E[(64 + rl) * 33 + q], w, old[x].y));
            }
          }
        }
        epi_sync();
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      epi_sync();
      if (threadIdx.x == 0) mbar_arrive(acce0 + 8 * (g & 1));
      g++;
    }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_d), "r"(2 * OZ_BN) : "memory");
}

// Tail tiles made of partial segments: tile fix[3 i] = the sum, in listed
// order, of workspace slots fix[3 j + 2] (= 2 CTA + slot) for the entries j of
// its run (fix[3 i + 1] = run length, given on the run's first entry)
__global__ void k_oz_fixup(const int64_t *__restrict__ fix, const int *__restrict__ runs, int ncol, int64_t M,
                           int64_t Rv, double2 *__restrict__ Y, const double2 *__restrict__ P, int64_t ldy) {
  const int j0 = runs[blockIdx.x];
  const int64_t t = fix[3 * j0], len = fix[3 * j0 + 1];
  const int64_t row0 = 64 * (t / ncol), col0 = (int64_t)OZ_BN * (t % ncol);
  for (int e = threadIdx.x; e < OZ_TILE_ELEMS; e += blockDim.x) {
    const int64_t r = row0 + (e & 63), c = col0 + (e >> 6);
    if (r >= M || c >= Rv) continue;
    double2 acc = make_double2(0, 0);
    for (int64_t j = 0; j < len; j++) acc = cadd(acc, P[fix[3 * (j0 + j) + 2] * OZ_TILE_ELEMS + e]);
    Y[c * ldy + r] = acc;
  }
}

// sigma (power of two, max/sigma in [0.5, 1)) of each complex row of Z
__global__ void k_oz_row_scale(int64_t N, const float2 *__restrict__ Z, double *__restrict__ rs) {
  __shared__ float red[8];
  const int64_t m = blockIdx.x;
  float mx = 0.f;
  for (int64_t k = threadIdx.x; k < N; k += blockDim.x) {
    const float2 z = Z[m * N + k];
    mx = fmaxf(mx, fmaxf(fabsf(z.x), fabsf(z.y)));
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) mx = fmaxf(mx, red[w]);
    int e = 0;
    frexp((double)mx, &e);
    rs[m] = mx > 0.f ? ldexp(1.0, e) : 1.0;
  }
}

// tau (power of two) of each column of X
__global__ void k_oz_col_scale(int64_t N, const double2 *__restrict__ X, double *__restrict__ cs) {
  __shared__ double red[8];
  const int64_t r = blockIdx.x;
  double mx = 0.0;
  for (int64_t k = threadIdx.x; k < N; k += blockDim.x) {
    const double2 x = X[r * N + k];
    mx = fmax(mx, fmax(fabs(x.x), fabs(x.y)));
  }
  mx = warp_max(mx);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) mx = fmax(mx, red[w]);
    int e = 0;
    frexp(mx, &e);
    cs[r] = mx > 0.0 ? ldexp(1.0, e) : 1.0;
  }
}

// next 7-bit slice of v in (-1, 1): a = trunc(128 v), v <- 128 v - a (exact)
__device__ __forceinline__ signed char oz_cut(double &v) {
  const double t = v * 128.0;
  const double a = trunc(t);
  v = t - a;
  return (signed char)(int)a;
}

// Z slices: slice p occupies rows [p 2Mpad, (p+1) 2Mpad); complex row m gives
// rows 128 (m/64) + m%64 ([Zr | -Zi]) and that + 64 ([Zi | Zr]); K'' = 2 Kh.
__global__ void k_oz_slice_a(int64_t N, int64_t Kh, int64_t Mpad, const float2 *__restrict__ Z,
                             const double *__restrict__ rs, signed char *__restrict__ A) {
  const int64_t m = blockIdx.y;
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= Kh) return;
  double ur = 0, ui = 0;
  if (m < N && k < N) {
    const float2 z = Z[m * N + k];
    const double inv = 1.0 / rs[m];  // power of two: exact
    ur = (double)z.x * inv;
    ui = (double)z.y * inv;
  }
  const int64_t ld = 2 * Kh, slice = 2 * Mpad * ld;
  const int64_t rr = 128 * (m / 64) + m % 64, ri = rr + 64;
#pragma unroll
  for (int p = 0; p < OZ_S; p++) {
    const signed char ar = oz_cut(ur), ai = oz_cut(ui);
    signed char *Ap = A + p * slice;
    Ap[rr * ld + k] = ar;
    Ap[rr * ld + Kh + k] = (signed char)(-ai);
    Ap[ri * ld + k] = ai;
    Ap[ri * ld + Kh + k] = ar;
  }
}

// X slices: slice q occupies rows [q Rpad, (q+1) Rpad); row r = [Xr | Xi]
__global__ void k_oz_slice_b(int64_t N, int64_t R, int64_t Kh, int64_t Rpad, const double2 *__restrict__ X,
                             const double *__restrict__ cs, signed char *__restrict__ B) {
  const int64_t r = blockIdx.y;
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= Kh) return;
  double ur = 0, ui = 0;
  if (r < R && k < N) {
    const double2 x = X[r * N + k];
    const double inv = 1.0 / cs[r];
    ur = x.x * inv;
    ui = x.y * inv;
  }
  const int64_t ld = 2 * Kh, slice = Rpad * ld;
#pragma unroll
  for (int q = 0; q < OZ_S; q++) {
    const signed char br = oz_cut(ur), bi = oz_cut(ui);
    signed char *Bq = B + q * slice;
    Bq[r * ld + k] = br;
    Bq[r * ld + Kh + k] = bi;
  }
}

int64_t round_up(int64_t v, int64_t m) { return ((v + m - 1) / m) * m; }
unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

struct OzState {
  DevBuf A, B, rs, cs, err, P, fix, runs;
  CUtensorMap mapA, mapB;
  uint64_t a_version = ~0ull;
  int64_t a_n = -1, b_key = -1, b_n = -1;
  bool attr = false;
};

std::mutex g_oz_mu;
std::vector<std::pair<dmb_ctx *, OzState *>> g_oz_states;

OzState &oz_state(dmb_ctx *c) {
  std::lock_guard<std::mutex> lk(g_oz_mu);
  for (auto &p : g_oz_states)
    if (p.first == c) return *p.second;
  g_oz_states.push_back({c, new OzState()});
  return *g_oz_states.back().second;
}

}  // namespace

namespace dmb {

// Is the int8 path usable for this Z (int32 headroom for at least one pair)?
bool oz_available(dmb_ctx *c) {
  if (!tc_available(c) || c->z_prec != DMB_PREC_MIXED) return false;
  const int64_t K = 2 * round_up(c->n, OZ_BK);
  return 16129.0 * (double)K < 2147483647.0;
}

// Slices of the current Z (row scales, six int8 slices, tensor map), made
// once per Z; may run on another stream ahead of the first product, which
// must then be ordered after it.
void oz_prepare(dmb_ctx *c) {
  DMB_REQUIRE(oz_available(c), DMB_ERR_STATE, "int8 tensor-core product unavailable for this matrix");
  OzState &st = oz_state(c);
  const int64_t N = c->n, Kh = round_up(N, OZ_BK), Mpad = round_up(N, 64);
  const int64_t ld = 2 * Kh;
  if (!st.err.p) {
    st.err.ensure(16);
    DMB_CUDA(cudaMemsetAsync(st.err.p, 0, 16, c->stream));
  }
  if (!st.attr) {
    DMB_CUDA(cudaFuncSetAttribute(k_oz_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, OZ_SMEM));
    st.attr = true;
  }
  if (st.a_version != c->z_version || st.a_n != N) {
    st.rs.ensure(sizeof(double) * Mpad);
    st.A.ensure((size_t)OZ_S * 2 * Mpad * ld);
    DMB_LAUNCH(c, k_oz_row_scale, (unsigned)N, 256, 0, N, c->d_Z.as<float2>(), st.rs.as<double>());
    DMB_LAUNCH(c, k_oz_slice_a, dim3(blocks_for(Kh, 256), (unsigned)Mpad), 256, 0, N, Kh, Mpad,
               c->d_Z.as<float2>(), st.rs.as<double>(), st.A.as<signed char>());
    make_map_bytes(&st.mapA, st.A.p, CU_TENSOR_MAP_DATA_TYPE_UINT8, (uint64_t)ld, (uint64_t)ld,
                   (uint64_t)(OZ_S * 2 * Mpad), OZ_BK, OZ_BM);
    st.a_version = c->z_version;
    st.a_n = N;
  }
}

void oz_zx(dmb_ctx *c, const double2 *X, double2 *Y, int64_t R, int lmax) {
  DMB_REQUIRE(lmax >= 0 && lmax <= OZ_LMAX, DMB_ERR_ARGUMENT, "int8 slice levels out of range");
  oz_prepare(c);
  OzState &st = oz_state(c);
  const int64_t N = c->n, Kh = round_up(N, OZ_BK), Mpad = round_up(N, 64), Rpad = round_up(R, OZ_BN);
  const int64_t ld = 2 * Kh;
  st.cs.ensure(sizeof(double) * Rpad);
  st.B.ensure((size_t)OZ_S * Rpad * ld);
  if (st.b_key != Rpad || st.b_n != N) {
    make_map_bytes(&st.mapB, st.B.p, CU_TENSOR_MAP_DATA_TYPE_UINT8, (uint64_t)ld, (uint64_t)ld,
                   (uint64_t)(OZ_S * Rpad), OZ_BK, OZ_BN);
    st.b_key = Rpad;
    st.b_n = N;
  }
  DMB_LAUNCH(c, k_oz_col_scale, (unsigned)R, 256, 0, N, X, st.cs.as<double>());
  DMB_LAUNCH(c, k_oz_slice_b, dim3(blocks_for(Kh, 256), (unsigned)Rpad), 256, 0, N, R, Kh, Rpad, X,
             st.cs.as<double>(), st.B.as<signed char>());
  // pair schedule: levels L = p + q <= OZ_LMAX, largest terms first; a level's
  // pairs share one TMEM sum unless int32 headroom forces an earlier drain
  const int64_t maxp = (int64_t)(2147483647.0 / (16129.0 * (double)ld));
  OzSched sc{};
  int n = 0;
  for (int L = 0; L <= lmax; L++) {
    int in_group = 0;
    for (int p = 0; p <= L; p++) {
      const int q = L - p;
      if (p >= OZ_S || q >= OZ_S) continue;
      sc.arow[n] = (int)(p * 2 * Mpad);
      sc.brow[n] = (int)(q * Rpad);
      sc.close[n] = 0;
      sc.lscale[n] = std::ldexp(1.0, -OZ_BETA * (L + 2));
      n++;
      if (++in_group == maxp) {
        sc.close[n - 1] = 1;
        in_group = 0;
      }
    }
    if (in_group > 0) sc.close[n - 1] = 1;
  }
  sc.n = n;
  // persistent grid: data-parallel full waves, stream-K tail (k_oz_gemm);
  // the host replays the tail split to list each partial tile's slots
  const int ncol = (int)(Rpad / OZ_BN);
  const int64_t ntiles = (Mpad / 64) * ncol;
  const int64_t G = std::min<int64_t>(ntiles, std::max(1, c->sm_count));
  const int64_t F = (ntiles / G) * G, Wt = (ntiles - F) * n;
  std::vector<int64_t> fix;  // (tile, run length, 2 CTA + slot) in tile order, then CTA order
  for (int64_t b = 0; b < G; b++) {
    int64_t u = F * n + Wt * b / G;
    const int64_t u_end = F * n + Wt * (b + 1) / G;
    int slot = 0;
    while (u < u_end) {
      const int64_t t = u / n;
      const int64_t p0 = u - t * n, p1 = std::min<int64_t>(n, u_end - t * n);
      u = t * n + p1;
      if (!(p0 == 0 && p1 == n)) fix.insert(fix.end(), {t, 0, 2 * b + slot++});
    }
  }
  std::vector<int> runs;
  for (size_t j = 0; j < fix.size() / 3; j++) {
    if (j == 0 || fix[3 * j] != fix[3 * (j - 1)]) runs.push_back((int)j);
    fix[3 * runs.back() + 1]++;
  }
  if (!fix.empty()) {
    st.P.ensure(sizeof(double2) * G * 2 * OZ_TILE_ELEMS);
    st.fix.ensure(sizeof(int64_t) * fix.size());
    st.runs.ensure(sizeof(int) * runs.size());
    DMB_CUDA(cudaMemcpyAsync(st.fix.p, fix.data(), sizeof(int64_t) * fix.size(), cudaMemcpyHostToDevice, c->stream));
    DMB_CUDA(cudaMemcpyAsync(st.runs.p, runs.data(), sizeof(int) * runs.size(), cudaMemcpyHostToDevice, c->stream));
  }
  kt_begin(c);
  DMB_LAUNCH(c, k_oz_gemm, (unsigned)G, 192, OZ_SMEM, st.mapA, st.mapB, sc, (int)(ld / OZ_BK), N, R, Y,
             fix.empty() ? Y : st.P.as<double2>(), N, ncol, ntiles, st.rs.as<double>(), st.cs.as<double>(),
             st.err.as<unsigned>());
  if (!runs.empty())
    DMB_LAUNCH(c, k_oz_fixup, (unsigned)runs.size(), 256, 0, st.fix.as<int64_t>(), st.runs.as<int>(), ncol, N, R,
               Y, st.P.as<double2>(), N);
  // int8 work: every kept slice pair is a real (2N x 2N) x (2N x R) product
  kt_end(c, 2.0 * n * (2.0 * N) * (2.0 * N) * (double)R, 1);
}

unsigned oz_error_word(dmb_ctx *c) {
  OzState &st = oz_state(c);
  if (!st.err.p) return 0;
  unsigned e = 0;
  DMB_CUDA(cudaMemcpyAsync(&e, st.err.p, 4, cudaMemcpyDeviceToHost, c->stream));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  return e;
}

void oz_release(dmb_ctx *c) {
  std::lock_guard<std::mutex> lk(g_oz_mu);
  for (size_t i = 0; i < g_oz_states.size(); i++) {
    if (g_oz_states[i].first != c) continue;
    OzState *st = g_oz_states[i].second;
    for (DevBuf *b : {&st->A, &st->B, &st->rs, &st->cs, &st->err, &st->P, &st->fix, &st->runs}) b->release();
    delete st;
    g_oz_states.erase(g_oz_states.begin() + i);
    return;
  }
}

}  // namespace dmb
