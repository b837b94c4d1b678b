// dmb_ozaki.cu -- FP64-accurate Y = Z X for a complex64 Z and complex128 X on
// the INT8 tensor cores (tcgen05.mma.kind::i8, exact int32 accumulation):
// the refinement and true residuals of the batched solves.
//
// Complex as one real product: row m of Z gives a real row [Zr, -Zi] and an
// imaginary row [Zi, Zr] against the column [Xr; Xi] (K = 2N).  Each complex
// row m of Z is scaled by sigma_m = 2^e (the smallest power of two above
// max_k max(|Zr|, |Zi|)), each column r of X by tau_r likewise.  Two ways of
// making the FP64-accurate product from exact int8 products:
//
// Residue scheme (default; the modular-arithmetic emulation of Ozaki, Uchino
// and Imamura, "Ozaki Scheme II: a GEMM-oriented emulation of floating-point
// matrix multiplication using an integer modular technique", 2025):
//   * the scaled values become integers A' = rint(2^a Z / sigma) and
//     B' = rint(2^b X / tau), |A'| <= 2^a, |B'| <= 2^b, with a + b chosen so
//     that the exact integer product C' = A' B' satisfies
//     K 2^(a + b) < M / 2, M the product of the moduli (13 pairwise coprime
//     moduli <= 256: M ~ 2^102.5, a = b = 43 at K = 21,504);
//   * per modulus m_i the symmetric residues A' mod m_i, B' mod m_i fit int8,
//     and their int8 product is exact in int32 (128^2 K < 2^31), so
//     C'_i = (A'_i B'_i) mod m_i = C' mod m_i;
//   * Chinese remainder theorem as a fraction: C' / M = sum_i C'_i y_i / m_i
//     (mod 1), y_i = (M / m_i)^-1 mod m_i.  The drains keep each C'_i (one
//     byte) in residue planes and the drain of a tile's last modulus forms
//     the 96-bit fixed-point fraction S = sum_i C'_i f_i (mod 2^96), f_i =
//     round(2^96 y_i / m_i), as a uint64 high word and a uint32 low word;
//     S / 2^96 is C' / M to within 2^-85, and
//     Y = (int64(hi) + lo 2^-32) M 2^-64 2^-(a + b) sigma tau.  (A 64-bit
//     fraction alone leaves ~2^-53 M of C', about 1e-12 of an EFIE row's
//     product.)  One int8 product per modulus: 13 for the residuals (~1e-13
//     normwise), 12 for the Krylov operator (b reduced by the missing modulus,
//     ~1e-11).  Integer sums are associative: every split of the moduli over
//     CTAs gives the same bits.
// Slice scheme (Ozaki, Ogita, Oishi & Rump, "Error-free transformations of
// matrix multiplication by using fast routines of matrix multiplication and
// its applications", Numer. Algorithms 59, 2012, with fixed-point int8
// slices):
//   * the scaled values in (-1, 1) are cut into OZ_S slices of OZ_BETA = 7
//     bits, v = sum_p a_p 2^(-7(p+1)) with integer a_p in [-127, 127] (exact in
//     double arithmetic);
//   * slice products a_p . b_q are exact in int32 (127^2 x 2N < 2^31 per pair);
//     pairs with p + q <= OZ_LMAX (0-based) are kept, summed in TMEM per level
//     (as many pairs per drain as int32 allows) and drained into FP64 with the
//     exact power-of-two weights sigma_m tau_r 2^(-7(L+2)).
//   With OZ_S = 6 and all levels up to OZ_LMAX = 6 (26 int8 products) the
//   product is ~7e-13 relative (normwise) on EFIE rows; the Krylov products
//   keep levels <= 5 (21 products, ~4e-11).
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
//   warps 0-3         drain each level (slices: tcgen05.ld, scale, FP64
//                     store / add); residues: warps 0-7 drain each modulus
//                     (tcgen05.ld, reduce mod m_i, one byte per element into
//                     the tile's residue planes; the last modulus of a tile
//                     reads the other residues back and converts to FP64).
// Every wait is bounded (error bit, abort flag, TMEM freed); every TMA load fills one CTA.
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

// pairwise coprime moduli, largest first (255 = 3 5 17, 253 = 11 23,
// 247 = 13 19, 217 = 7 31, the rest prime)
constexpr int OZ_NMOD = 13;
constexpr int OZ_MODULI[OZ_NMOD] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211};

struct OzSched {
  int n;
  int arow[OZ_MAXP];      // first A'' row of the pair's Z slice / residue plane
  int brow[OZ_MAXP];      // first B'' row of the pair's X slice / residue plane
  int close[OZ_MAXP];     // 1: the TMEM sum is drained after this pair
  double lscale[OZ_MAXP]; // slices: weight of the pair's level, 2^(-7 (L + 2))
  // residues: modulus, reduction constants (oz_mod), CRT fraction
  // round(2^96 y_i / m_i) as high 64 and low 32 bits
  int mod[OZ_MAXP];
  unsigned mmul[OZ_MAXP], moff[OZ_MAXP];
  unsigned long long frac[OZ_MAXP];
  unsigned fraclo[OZ_MAXP];
  double cscale;          // residues: M 2^-64 2^-(a + b)
};

// v mod m in [0, m) for an int8-product sum |v| <= 2^31 - 2^14 and
// 199 <= m <= 256, in integer arithmetic: u = v + moff (moff = m
// floor(2^31 / m), so 0 < u < 2^32 and u = v mod m), q = floor(u mmul /
// 2^39) with mmul = ceil(2^39 / m) is floor(u / m) or one more (the error of
// u mmul / 2^39 is below u / 2^39 < 2^-7), one correction.
__device__ __forceinline__ unsigned oz_mod(int v, unsigned m, unsigned mmul, unsigned moff) {
  const unsigned u = (unsigned)v + moff;
  const unsigned q = __umulhi(u, mmul) >> 7;
  const int r = (int)(u - q * m);
  return (unsigned)(r < 0 ? r + (int)m : r);
}

// Global accesses to the residue planes marked evict-last in L2: a CTA's
// planes (416 KB) are read back at its tile's last modulus, while the int8
// operand planes stream through L2 once per product.
__device__ __forceinline__ uint64_t l2_evict_last_policy() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint4 ld_keep4(const uint4 *a, uint64_t pol) {
  uint4 v;
  asm volatile("ld.global.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ void st_keep4(uint4 *a, uint4 v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v4.u32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(a), "r"(v.x), "r"(v.y),
               "r"(v.z), "r"(v.w), "l"(pol)
               : "memory");
}

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
// residues of one tile: OZ_NMOD planes of 128 real-stacked rows x 256 columns,
// one byte each; in a plane, 16-column groups of 128 rows x 16 bytes (row r's
// 16 residues of group g at byte g 2048 + 16 r)
constexpr int OZ_RES_PLANE = 128 * OZ_BN;
constexpr int64_t OZ_RES_TILE = (int64_t)OZ_NMOD * OZ_RES_PLANE;

// S = sum over the 16 residues packed in p (bytes, element q in byte q) of
// r_q f, f = fh 2^32 + fl, accumulated as th 2^32 + tl (tl < 2^44 for up to
// 13 terms, so no carry is lost before the final fold)
__device__ __forceinline__ void oz_frac_add(const uint4 p, unsigned long long fh, unsigned long long fl,
                                            unsigned long long (&th)[16], unsigned long long (&tl)[16]) {
  const unsigned w[4] = {p.x, p.y, p.z, p.w};
#pragma unroll
  for (int q = 0; q < 16; q++) {
    const unsigned long long u = (w[q >> 2] >> (8 * (q & 3))) & 0xffu;
    tl[q] += u * fl;
    th[q] += u * fh;
  }
}

// warps per CTA: slices 4 drain + producer + MMA issuer; residues 8 drain
// (two per TMEM lane quarter, each on half of the columns) + producer + MMA
template <bool CRT> constexpr int oz_threads() { return CRT ? 320 : 192; }

template <bool CRT>
__global__ void __launch_bounds__(oz_threads<CRT>(), 1) k_oz_gemm(const __grid_constant__ CUtensorMap tmA,
                                                    const __grid_constant__ CUtensorMap tmB,
                                                    const __grid_constant__ OzSched sc, int kchunks, int64_t M,
                                                    int64_t Rv, double2 *__restrict__ Y, double2 *__restrict__ P,
                                                    int64_t ldy, int ncol, int64_t ntiles,
                                                    const double *__restrict__ rs, const double *__restrict__ cs,
                                                    unsigned char *__restrict__ Rres, unsigned *err) {

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
      mbar_init(acce0 + 8 * b, CRT ? 8 : 1);  // residues: one arrival per drain warp
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

  constexpr int W_PROD = CRT ? 8 : 4, W_MMA = CRT ? 9 : 5;
  if (warp == W_PROD) {
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
  } else if (warp == W_MMA) {
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
  } else if (CRT) {
    // residue drains: each of warps 0-7 works alone on the 32 TMEM lanes =
    // tile rows of its quarter (warp & 3; rows 0-63: real parts of the 64
    // complex rows, 64-127: imaginary parts) and on half of the columns
    // (warp >> 2).  Per modulus a thread reads its row's int32 sums, 16
    // columns at a time, reduces them mod m_i and stores the 16 residues as
    // one 16-byte word into the tile's plane i (a warp writes 512 contiguous
    // bytes).  The last modulus of a whole tile instead reads the other
    // planes' words of the same 16 elements back, forms the CRT fraction and
    // writes Y.  Whole tiles use the CTA's own planes; tail tiles (split
    // stream-K over CTAs) have planes of their own and are converted by
    // k_oz_fixup.  Each warp arrives on the accumulator-empty barrier by
    // itself (count 8).
    const int row = (warp & 3) * 32 + lane;
    const int chalf = warp >> 2;
    const uint64_t keep = l2_evict_last_policy();
    const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
    const int64_t ftile = (ntiles / gridDim.x) * gridDim.x;  // the first tail tile
    int g = 0;
    bool alive = true;
    OzIter it;
    oz_iter_init(it, ntiles, sc.n);
    OzSeg sg;
    while (alive && oz_next_seg(it, sg)) {
      const int64_t row0 = 64 * (sg.t / ncol), col0 = (int64_t)OZ_BN * (sg.t % ncol);
      const bool tail = sg.t >= ftile;
      const int64_t rt = tail ? (int64_t)gridDim.x + (sg.t - ftile) : (int64_t)blockIdx.x;
      uint4 *Rt = reinterpret_cast<uint4 *>(Rres + rt * OZ_RES_TILE) + row;
      const int64_t gr = row0 + (row & 63);
      const bool row_ok = gr < M;
      const double rsc = row_ok ? rs[gr] * sc.cscale : 0.0;
      // this warp's 16-column groups that hold data
      const int cc0 = chalf * (OZ_BN / 32);
      const int cc1 = (int)min((int64_t)(cc0 + OZ_BN / 32), (Rv - col0 + 15) / 16);
      for (int i = sg.p0; i < sg.p1; i++) {
        const bool fin = !tail && i + 1 == sc.n;
        const unsigned gm = (unsigned)sc.mod[i], gmul = sc.mmul[i], goff = sc.moff[i];
        // warp-uniform outcome: the loads below are warp-collective
        const bool got = mbar_wait(accf0 + 8 * (g & 1), (uint32_t)(g >> 1) & 1u, err, abort_flag);
        if (!__all_sync(0xffffffffu, got)) {
          alive = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t tacc = tmem_d + (uint32_t)((g & 1) * OZ_BN) + lane_base;
        for (int cc = cc0; cc < cc1; cc++) {
          uint32_t v[16];
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
              : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                "=r"(v[15])
              : "r"(tacc + (uint32_t)(cc * 16)));
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          unsigned w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
          for (int q = 0; q < 16; q++) w[q >> 2] |= oz_mod((int)v[q], gm, gmul, goff) << (8 * (q & 3));
          if (!fin) {
            st_keep4(Rt + i * (OZ_RES_PLANE / 16) + cc * 128, make_uint4(w[0], w[1], w[2], w[3]), keep);
            continue;
          }
          unsigned long long th[16], tl[16];
#pragma unroll
          for (int q = 0; q < 16; q++) th[q] = tl[q] = 0ull;
          for (int j = 0; j < i; j++)
            oz_frac_add(ld_keep4(Rt + j * (OZ_RES_PLANE / 16) + cc * 128, keep), sc.frac[j], sc.fraclo[j], th, tl);
          oz_frac_add(make_uint4(w[0], w[1], w[2], w[3]), sc.frac[i], sc.fraclo[i], th, tl);
          if (row_ok) {
#pragma unroll
            for (int q = 0; q < 16; q++) {
              const int64_t c = col0 + cc * 16 + q;
              const unsigned long long hi = th[q] + (tl[q] >> 32);
              if (c < Rv)
                reinterpret_cast<double *>(Y)[2 * (c * ldy + gr) + (row >> 6)] =
                    fma((double)(unsigned)tl[q], 0x1p-32, (double)(long long)hi) * rsc * cs[c];
            }
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(acce0 + 8 * (g & 1));
        g++;
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

// ---------------------------------------------------------------------------
// Residue scheme on CTA pairs (tcgen05 cta_group::2): a cluster of two CTAs
// on one TPC computes a 128 x 256 complex tile (256 real-stacked rows) as one
// M = 256, N = 256 int8 MMA per K step, issued by the even CTA.  Each CTA
// loads its own 128 A rows and half of the 256 B rows (plain TMA tile loads
// into its own shared memory, both completing on the even CTA's full
// barrier), so per int8 MAC an SM reads a third less operand data than with
// the one-SM 128 x 256 tile.  The accumulator rows of each CTA sit in its own
// TMEM (rows 0-127 even, 128-255 odd CTA, all 256 columns), so each CTA
// drains its 64 complex rows exactly as k_oz_gemm does (residue planes, CRT
// at the last modulus).  The MMA's commits arrive on the barriers of both
// CTAs (one commit, two-CTA mask); the odd CTA's drain warps arrive on the
// even CTA's accumulator-empty barrier.  Every wait is bounded (error bit 8,
// per-CTA abort flag, TMEM freed).  Measured on the headline product it runs
// at the same tensor-pipe activity as the one-SM tile (68 %) and is not
// faster (4.7-4.8 vs 4.25 ms): the launch is bound by the int8 MMA issue
// under the power cap, not by the operand feed; the autotuner keeps it as a
// candidate.
constexpr int OZP_STAGES = 6;
constexpr int OZP_A_STAGE = 128 * OZ_BK, OZP_B_STAGE = 128 * OZ_BK;  // per CTA
constexpr int OZP_SMEM = OZP_STAGES * (OZP_A_STAGE + OZP_B_STAGE) + 256 /*barriers*/ + 1024 /*align*/;
// D s32, A/B signed int8, K-major, N = 256, M = 256 (the pair)
constexpr uint32_t OZP_IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(256 >> 3) << 17) |
                               ((uint32_t)(256 >> 4) << 24);

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// shared::cluster address of the even CTA's copy of a local shared address
__device__ __forceinline__ uint32_t to_even_cta(uint32_t saddr) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(0u));
  return r;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// TMA tile load into this CTA's shared memory, completing on an mbarrier of
// either CTA of the pair
__device__ __forceinline__ void tma_load_2d_pair(uint32_t dst, const CUtensorMap *map, int x, int y,
                                                 uint32_t bar_cluster) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
      "%3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar_cluster)
      : "memory");
}
__device__ __forceinline__ void umma_i8_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(OZP_IDESC), "r"(accumulate)
      : "memory");
}
// arrive (once per CTA) on the barrier at this offset in both CTAs of the
// pair when the MMAs issued so far have completed
__device__ __forceinline__ void umma_commit_pair(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(bar),
      "h"((unsigned short)3)
      : "memory");
}
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t bar_cluster) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar_cluster) : "memory");
}
// bounded wait with cluster-scope acquire (arrivals from the other CTA)
__device__ __forceinline__ bool mbar_wait_cluster(uint32_t bar, uint32_t parity, unsigned *err,
                                                  volatile int *abort) {
  for (long long it = 0; it < TC_WAIT_LIMIT; it++) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    if ((it & 1023) == 1023 && *abort) return false;
  }
  atomicOr(err, 8u);
  *abort = 1;
  return false;
}

// work of cluster b of G over npairs pair tiles: whole pair tiles in
// data-parallel waves, the tail split stream-K as in k_oz_gemm
__device__ __forceinline__ void oz_iter_init_pair(OzIter &it, int64_t npairs, int n) {
  it.G = gridDim.x / 2;
  it.b = blockIdx.x / 2;
  it.n = n;
  it.wave = 0;
  it.nfull = npairs / it.G;
  const int64_t F = it.nfull * it.G, Wt = (npairs - F) * n;
  it.u = F * n + Wt * it.b / it.G;
  it.u_end = F * n + Wt * (it.b + 1) / it.G;
  it.slot = 0;
}

__global__ void __launch_bounds__(320, 1) k_oz_pair(const __grid_constant__ CUtensorMap tmA,
                                                    const __grid_constant__ CUtensorMap tmB,
                                                    const __grid_constant__ OzSched sc, int kchunks, int64_t M,
                                                    int64_t Rv, double2 *__restrict__ Y, int64_t ldy, int ncol,
                                                    int64_t npairs, const double *__restrict__ rs,
                                                    const double *__restrict__ cs, unsigned char *__restrict__ Rres,
                                                    unsigned *err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char *gbase = smem_raw + (base - raw);
  const uint32_t sA = base;
  const uint32_t sB = base + OZP_STAGES * OZP_A_STAGE;
  const uint32_t sBar = sB + OZP_STAGES * OZP_B_STAGE;
  uint64_t *bar_ptr = reinterpret_cast<uint64_t *>(gbase + (sBar - base));
  volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(bar_ptr + 20);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(bar_ptr + 21);
  // full[s] (even CTA: both CTAs' loads), empty[s] (each CTA: its stage
  // consumed), accf[b] (each CTA: accumulator b full), acce[b] (even CTA:
  // accumulator b drained by both CTAs, 16 warp arrivals)
  const uint32_t full0 = sBar, empty0 = sBar + 8 * OZP_STAGES, accf0 = sBar + 16 * OZP_STAGES, acce0 = accf0 + 16;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();
  if (threadIdx.x == 0) {
    for (int s = 0; s < OZP_STAGES; s++) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(accf0 + 8 * b, 1);
      mbar_init(acce0 + 8 * b, 16);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(const_cast<uint32_t *>(tmem_slot))),
                 "r"(2 * OZ_BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  // both CTAs' barriers initialised and TMEM allocated before any use
  cluster_sync_all();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem_d = *tmem_slot;

  if (warp == 8) {
    if (lane == 0) {
      const uint32_t full_even = to_even_cta(full0);
      long long t = 0;
      OzIter it;
      oz_iter_init_pair(it, npairs, sc.n);
      OzSeg sg;
      bool go = true;
      while (go && oz_next_seg(it, sg)) {
        // this CTA's 128 A rows and 128 B rows of the pair tile
        const int arow = (int)(256 * (sg.t / ncol) + 128 * rank);
        const int brow = (int)(OZ_BN * (sg.t % ncol) + 128 * rank);
        for (int i = sg.p0; i < sg.p1 && go; i++) {
          for (int kc = 0; kc < kchunks; kc++, t++) {
            const int s = (int)(t % OZP_STAGES);
            if (*abort_flag || (t >= OZP_STAGES && !mbar_wait(empty0 + 8 * s, (uint32_t)((t / OZP_STAGES) - 1) & 1u,
                                                              err, abort_flag))) {
              go = false;
              break;
            }
            if (rank == 0) mbar_expect_tx(full0 + 8 * s, 2 * (OZP_A_STAGE + OZP_B_STAGE));
            tma_load_2d_pair(sA + s * OZP_A_STAGE, &tmA, kc * OZ_BK, sc.arow[i] + arow, full_even + 8 * s);
            tma_load_2d_pair(sB + s * OZP_B_STAGE, &tmB, kc * OZ_BK, sc.brow[i] + brow, full_even + 8 * s);
          }
        }
      }
    }
  } else if (warp == 9) {
    if (lane == 0 && rank == 0) {
      long long t = 0;
      int g = 0;
      bool ok = true;
      OzIter it;
      oz_iter_init_pair(it, npairs, sc.n);
      OzSeg sg;
      while (ok && oz_next_seg(it, sg)) {
        for (int i = sg.p0; i < sg.p1 && ok; i++) {
          // modulus g accumulates in buffer g & 1, free once modulus g - 2 is
          // drained by both CTAs
          if (g >= 2 && !mbar_wait_cluster(acce0 + 8 * (g & 1), (uint32_t)((g >> 1) - 1) & 1u, err, abort_flag)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t tmem_acc = tmem_d + (uint32_t)((g & 1) * OZ_BN);
          for (int kc = 0; kc < kchunks; kc++, t++) {
            const int s = (int)(t % OZP_STAGES);
            if (!mbar_wait(full0 + 8 * s, (uint32_t)(t / OZP_STAGES) & 1u, err, abort_flag)) {
              ok = false;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int k = 0; k < OZ_BK / 32; k++) {
              const uint64_t ad = sw128_desc(sA + s * OZP_A_STAGE + k * 32);
              const uint64_t bd = sw128_desc(sB + s * OZP_B_STAGE + k * 32);
              umma_i8_pair(tmem_acc, ad, bd, (kc == 0 && k == 0) ? 0u : 1u);
            }
            umma_commit_pair(empty0 + 8 * s);
          }
          if (ok) umma_commit_pair(accf0 + 8 * (g & 1));
          g++;
        }
      }
    }
  } else {
    // residue drains of this CTA's 64 complex rows (as in k_oz_gemm)
    const int row = (warp & 3) * 32 + lane;
    const int chalf = warp >> 2;
    const uint64_t keep = l2_evict_last_policy();
    const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
    const uint32_t acce_even = to_even_cta(acce0);
    const int64_t G2 = gridDim.x / 2;
    const int64_t fpair = (npairs / G2) * G2;  // the first tail pair tile
    int g = 0;
    bool alive = true;
    OzIter it;
    oz_iter_init_pair(it, npairs, sc.n);
    OzSeg sg;
    while (alive && oz_next_seg(it, sg)) {
      const int64_t prow = sg.t / ncol;
      const int64_t row0 = 128 * prow + 64 * rank, col0 = (int64_t)OZ_BN * (sg.t % ncol);
      const bool tail = sg.t >= fpair;
      const int64_t rt = tail ? 2 * G2 + 2 * (sg.t - fpair) + rank : (int64_t)blockIdx.x;
      uint4 *Rt = reinterpret_cast<uint4 *>(Rres + rt * OZ_RES_TILE) + row;
      const int64_t gr = row0 + (row & 63);
      const bool row_ok = gr < M;
      const double rsc = row_ok ? rs[gr] * sc.cscale : 0.0;
      const int cc0 = chalf * (OZ_BN / 32);
      const int cc1 = (int)min((int64_t)(cc0 + OZ_BN / 32), (Rv - col0 + 15) / 16);
      for (int i = sg.p0; i < sg.p1; i++) {
        const bool fin = !tail && i + 1 == sc.n;
        const unsigned gm = (unsigned)sc.mod[i], gmul = sc.mmul[i], goff = sc.moff[i];
        const bool got = mbar_wait(accf0 + 8 * (g & 1), (uint32_t)(g >> 1) & 1u, err, abort_flag);
        if (!__all_sync(0xffffffffu, got)) {
          alive = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t tacc = tmem_d + (uint32_t)((g & 1) * OZ_BN) + lane_base;
        for (int cc = cc0; cc < cc1; cc++) {
          uint32_t v[16];
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
              : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                "=r"(v[15])
              : "r"(tacc + (uint32_t)(cc * 16)));
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          unsigned w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
          for (int q = 0; q < 16; q++) w[q >> 2] |= oz_mod((int)v[q], gm, gmul, goff) << (8 * (q & 3));
          if (!fin) {
            st_keep4(Rt + i * (OZ_RES_PLANE / 16) + cc * 128, make_uint4(w[0], w[1], w[2], w[3]), keep);
            continue;
          }
          unsigned long long th[16], tl[16];
#pragma unroll
          for (int q = 0; q < 16; q++) th[q] = tl[q] = 0ull;
          for (int j = 0; j < i; j++)
            oz_frac_add(ld_keep4(Rt + j * (OZ_RES_PLANE / 16) + cc * 128, keep), sc.frac[j], sc.fraclo[j], th, tl);
          oz_frac_add(make_uint4(w[0], w[1], w[2], w[3]), sc.frac[i], sc.fraclo[i], th, tl);
          if (row_ok) {
#pragma unroll
            for (int q = 0; q < 16; q++) {
              const int64_t c = col0 + cc * 16 + q;
              const unsigned long long hi = th[q] + (tl[q] >> 32);
              if (c < Rv)
                reinterpret_cast<double *>(Y)[2 * (c * ldy + gr) + (row >> 6)] =
                    fma((double)(unsigned)tl[q], 0x1p-32, (double)(long long)hi) * rsc * cs[c];
            }
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive_cluster(acce_even + 8 * (g & 1));
        g++;
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  // neither CTA frees TMEM or exits while the other may still use its
  // barriers or the MMA may still write its accumulators
  cluster_sync_all();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_d), "r"(2 * OZ_BN) : "memory");
}

// Tail tiles made of partial segments (slice scheme): tile fix[3 i] = the
// sum, in listed order, of workspace slots fix[3 j + 2] (= 2 CTA + slot) for
// the entries j of its run (fix[3 i + 1] = run length, given on the run's
// first entry)
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

// Tail tiles of the residue scheme: every modulus was drained into the
// tile's own residue planes (G + blockIdx.x), by whichever CTAs computed it;
// each element's residues are read back and converted to FP64 as the last
// drain of a whole tile does (the same integer sum, so the same bits).  One
// CTA per 64 x 256 tile: tile ftile + blockIdx.x of k_oz_gemm, or (pair)
// half blockIdx.x & 1 of pair tile ftile + blockIdx.x / 2 of k_oz_pair.
__global__ void __launch_bounds__(256) k_oz_crt_tail(const __grid_constant__ OzSched sc, int ncol, int64_t M,
                                                     int64_t Rv, int64_t ftile, int G, int pair,
                                                     double2 *__restrict__ Y, int64_t ldy,
                                                     const double *__restrict__ rs, const double *__restrict__ cs,
                                                     const unsigned char *__restrict__ Rres) {
  const int64_t t = pair ? ftile + blockIdx.x / 2 : ftile + blockIdx.x;
  const int64_t row0 = pair ? 128 * (t / ncol) + 64 * (blockIdx.x & 1) : 64 * (t / ncol);
  const int64_t col0 = (int64_t)OZ_BN * (t % ncol);
  const uint4 *Rt = reinterpret_cast<const uint4 *>(Rres + ((int64_t)G + blockIdx.x) * OZ_RES_TILE);
  for (int e = threadIdx.x; e < 128 * (OZ_BN / 16); e += blockDim.x) {
    const int row = e & 127, cc = e >> 7;  // consecutive threads: consecutive rows
    const int64_t gr = row0 + (row & 63);
    if (gr >= M || col0 + cc * 16 >= Rv) continue;
    unsigned long long th[16], tl[16];
#pragma unroll
    for (int q = 0; q < 16; q++) th[q] = tl[q] = 0ull;
    for (int j = 0; j < sc.n; j++)
      oz_frac_add(Rt[j * (OZ_RES_PLANE / 16) + cc * 128 + row], sc.frac[j], sc.fraclo[j], th, tl);
    const double rsc = rs[gr] * sc.cscale;
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const int64_t c = col0 + cc * 16 + q;
      const unsigned long long hi = th[q] + (tl[q] >> 32);
      if (c < Rv)
        reinterpret_cast<double *>(Y)[2 * (c * ldy + gr) + (row >> 6)] =
            fma((double)(unsigned)tl[q], 0x1p-32, (double)(long long)hi) * rsc * cs[c];
    }
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

// the first n moduli and their reciprocals, for the residue kernels
struct OzMods {
  int n;
  double m[OZ_NMOD], minv[OZ_NMOD];
};

// symmetric residue of the integer-valued a (|a| < 2^52) modulo m, as int8:
// [-(m-1)/2, (m-1)/2] for odd m, [-128, 127] for m = 256
__device__ __forceinline__ int oz_res(double a, double m, double minv) {
  const double q = rint(a * minv);
  double r = fma(-q, m, a);  // exact: a - q m is an integer of a few bits
  if (r > 0.5 * m) r -= m;
  else if (r < -0.5 * m) r += m;
  const int v = (int)r;
  return v == 128 ? -128 : v;
}
__device__ __forceinline__ int oz_neg8(int v) { return v == -128 ? -128 : -v; }  // -(-128) = 128 = -128 mod 256
__device__ __forceinline__ uint32_t oz_pack4(int a, int b, int c, int d) {
  return (uint32_t)(a & 255) | ((uint32_t)(b & 255) << 8) | ((uint32_t)(c & 255) << 16) | ((uint32_t)(d & 255) << 24);
}

// Z residue planes: plane i occupies rows [i 2Mpad, (i+1) 2Mpad) in the layout
// of the slices (complex row m -> rows 128 (m/64) + m%64 ([Zr | -Zi]) and that
// + 64 ([Zi | Zr])), entries A' mod m_i with A' = rint(2^a Z / sigma_m).  One
// thread per 16 consecutive k (16-byte stores).
__global__ void __launch_bounds__(128) k_oz_res_a(int64_t N, int64_t Kh, int64_t Mpad, const float2 *__restrict__ Z,
                                                  const double *__restrict__ rs, double two_a, OzMods md,
                                                  signed char *__restrict__ A) {
  const int64_t m = blockIdx.y;
  const int64_t k0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * 16;
  if (k0 >= Kh) return;
  const double sc = m < N ? two_a / rs[m] : 0.0;  // power of two: exact
  double ar[16], ai[16];
#pragma unroll
  for (int u = 0; u < 16; u++) {
    const int64_t k = k0 + u;
    const float2 z = (m < N && k < N) ? Z[m * N + k] : make_float2(0.f, 0.f);
    ar[u] = rint((double)z.x * sc);
    ai[u] = rint((double)z.y * sc);
  }
  const int64_t ld = 2 * Kh, plane = 2 * Mpad * ld;
  const int64_t rr = 128 * (m / 64) + m % 64, ri = rr + 64;
  for (int i = 0; i < md.n; i++) {
    int pr[16], pi[16];
#pragma unroll
    for (int u = 0; u < 16; u++) {
      pr[u] = oz_res(ar[u], md.m[i], md.minv[i]);
      pi[u] = oz_res(ai[u], md.m[i], md.minv[i]);
    }
    uint4 vr, vni, vi;
    vr = make_uint4(oz_pack4(pr[0], pr[1], pr[2], pr[3]), oz_pack4(pr[4], pr[5], pr[6], pr[7]),
                    oz_pack4(pr[8], pr[9], pr[10], pr[11]), oz_pack4(pr[12], pr[13], pr[14], pr[15]));
    vi = make_uint4(oz_pack4(pi[0], pi[1], pi[2], pi[3]), oz_pack4(pi[4], pi[5], pi[6], pi[7]),
                    oz_pack4(pi[8], pi[9], pi[10], pi[11]), oz_pack4(pi[12], pi[13], pi[14], pi[15]));
    vni = make_uint4(oz_pack4(oz_neg8(pi[0]), oz_neg8(pi[1]), oz_neg8(pi[2]), oz_neg8(pi[3])),
                     oz_pack4(oz_neg8(pi[4]), oz_neg8(pi[5]), oz_neg8(pi[6]), oz_neg8(pi[7])),
                     oz_pack4(oz_neg8(pi[8]), oz_neg8(pi[9]), oz_neg8(pi[10]), oz_neg8(pi[11])),
                     oz_pack4(oz_neg8(pi[12]), oz_neg8(pi[13]), oz_neg8(pi[14]), oz_neg8(pi[15])));
    signed char *Ap = A + i * plane;
    *reinterpret_cast<uint4 *>(Ap + rr * ld + k0) = vr;
    *reinterpret_cast<uint4 *>(Ap + rr * ld + Kh + k0) = vni;
    *reinterpret_cast<uint4 *>(Ap + ri * ld + k0) = vi;
    *reinterpret_cast<uint4 *>(Ap + ri * ld + Kh + k0) = vr;
  }
}

// X residue planes: plane i occupies rows [i Rpad, (i+1) Rpad); row r =
// [Xr | Xi] mod m_i with B' = rint(2^b X / tau_r)
__global__ void __launch_bounds__(128) k_oz_res_b(int64_t N, int64_t R, int64_t Kh, int64_t Rpad,
                                                  const double2 *__restrict__ X, const double *__restrict__ cs,
                                                  double two_b, OzMods md, signed char *__restrict__ B) {
  const int64_t r = blockIdx.y;
  const int64_t k0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * 16;
  if (k0 >= Kh) return;
  const double sc = r < R ? two_b / cs[r] : 0.0;
  double br[16], bi[16];
#pragma unroll
  for (int u = 0; u < 16; u++) {
    const int64_t k = k0 + u;
    const double2 x = (r < R && k < N) ? X[r * N + k] : make_double2(0.0, 0.0);
    br[u] = rint(x.x * sc);
    bi[u] = rint(x.y * sc);
  }
  const int64_t ld = 2 * Kh, plane = Rpad * ld;
  for (int i = 0; i < md.n; i++) {
    int pr[16], pi[16];
#pragma unroll
    for (int u = 0; u < 16; u++) {
      pr[u] = oz_res(br[u], md.m[i], md.minv[i]);
      pi[u] = oz_res(bi[u], md.m[i], md.minv[i]);
    }
    signed char *Bp = B + i * plane + r * ld;
    *reinterpret_cast<uint4 *>(Bp + k0) =
        make_uint4(oz_pack4(pr[0], pr[1], pr[2], pr[3]), oz_pack4(pr[4], pr[5], pr[6], pr[7]),
                   oz_pack4(pr[8], pr[9], pr[10], pr[11]), oz_pack4(pr[12], pr[13], pr[14], pr[15]));
    *reinterpret_cast<uint4 *>(Bp + Kh + k0) =
        make_uint4(oz_pack4(pi[0], pi[1], pi[2], pi[3]), oz_pack4(pi[4], pi[5], pi[6], pi[7]),
                   oz_pack4(pi[8], pi[9], pi[10], pi[11]), oz_pack4(pi[12], pi[13], pi[14], pi[15]));
  }
}

// Host side of the residue scheme: exponents a (Z) and b (X) and the CRT
// constants of the first nm moduli.  The exact integer product C' needs
// K 2^(a + b) < M / 2, checked in 128-bit integers.
struct CrtConst {
  unsigned __int128 M = 1;
  double log2M = 0;
  unsigned long long frac[OZ_NMOD];
  unsigned fraclo[OZ_NMOD];
};
CrtConst crt_const(int nm) {
  CrtConst k;
  for (int i = 0; i < nm; i++) {
    k.M *= (unsigned)OZ_MODULI[i];
    k.log2M += std::log2((double)OZ_MODULI[i]);
  }
  for (int i = 0; i < nm; i++) {
    const int mi = OZ_MODULI[i];
    int Mi = 1;  // (M / m_i) mod m_i
    for (int j = 0; j < nm; j++)
      if (j != i) Mi = (Mi * (OZ_MODULI[j] % mi)) % mi;
    int y = 1;
    while ((Mi * y) % mi != 1) y++;  // m_i <= 256: direct search
    const unsigned __int128 f = (((unsigned __int128)y << 96) + (unsigned)(mi / 2)) / (unsigned)mi;  // < 2^96
    k.frac[i] = (unsigned long long)(f >> 32);
    k.fraclo[i] = (unsigned)(f & 0xffffffffu);
  }
  return k;
}
bool crt_fits(int64_t K, int e, const CrtConst &k) {  // K 2^e < M / 2
  return e >= 0 && e <= 100 && ((unsigned __int128)K << (e + 1)) < k.M;  // K < 2^18
}
int crt_exp_a(int64_t K) {  // a = b for all moduli
  const CrtConst k = crt_const(OZ_NMOD);
  int a = (int)std::floor((k.log2M - 1.0 - std::log2((double)K)) / 2.0);
  a = std::min(a, 52);
  while (a > 0 && !crt_fits(K, 2 * a, k)) a--;
  return a;
}
int crt_exp_b(int64_t K, int a, const CrtConst &k) {
  int b = (int)std::floor(k.log2M - 1.0 - std::log2((double)K)) - a;
  b = std::min(b, 52);
  while (b > 0 && !crt_fits(K, a + b, k)) b--;
  return b;
}
OzMods oz_mods(int nm) {
  OzMods md{};
  md.n = nm;
  for (int i = 0; i < OZ_NMOD; i++) {
    md.m[i] = OZ_MODULI[i];
    md.minv[i] = 1.0 / OZ_MODULI[i];
  }
  return md;
}

int64_t round_up(int64_t v, int64_t m) { return ((v + m - 1) / m) * m; }
unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

struct OzState {
  DevBuf A, B, rs, cs, err, P, fix, runs, Rres;
  CUtensorMap mapA, mapB, mapB128;
  uint64_t a_version = ~0ull;
  int64_t a_n = -1, b_key = -1, b_n = -1;
  int a_scheme = -1, b_scheme = -1;
  int crt_a = 0;  // residues: the Z exponent a of the current planes
  bool attr = false, pair_attr = false;
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

// Is the int8 path usable for this Z (int32 headroom for one product of
// int8 operands: |slice| <= 127, |residue| <= 128)?
bool oz_available(dmb_ctx *c) {
  if (!tc_available(c) || c->z_prec != DMB_PREC_MIXED) return false;
  const int64_t K = 2 * round_up(c->n, OZ_BK);
  return (c->int8_scheme == 0 ? 16384.0 : 16129.0) * (double)K < 2147483647.0;
}

// Operand planes of the current Z (row scales, int8 residues or slices,
// tensor map), made once per Z; may run on another stream ahead of the first
// product, which must then be ordered after it.
void oz_prepare(dmb_ctx *c) {
  DMB_REQUIRE(oz_available(c), DMB_ERR_STATE, "int8 tensor-core product unavailable for this matrix");
  OzState &st = oz_state(c);
  const int64_t N = c->n, Kh = round_up(N, OZ_BK), Mpad = round_up(N, 128);
  const int64_t ld = 2 * Kh;
  const bool crt = c->int8_scheme == 0;
  const int planes = crt ? OZ_NMOD : OZ_S;
  if (!st.err.p) {
    st.err.ensure(16);
    DMB_CUDA(cudaMemsetAsync(st.err.p, 0, 16, c->stream));
  }
  if (!st.attr) {
    DMB_CUDA(cudaFuncSetAttribute(k_oz_gemm<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, OZ_SMEM));
    DMB_CUDA(cudaFuncSetAttribute(k_oz_gemm<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, OZ_SMEM));
    st.attr = true;
  }
  if (st.a_version != c->z_version || st.a_n != N || st.a_scheme != c->int8_scheme) {
    st.rs.ensure(sizeof(double) * Mpad);
    st.A.ensure((size_t)planes * 2 * Mpad * ld);
    DMB_LAUNCH(c, k_oz_row_scale, (unsigned)N, 256, 0, N, c->d_Z.as<float2>(), st.rs.as<double>());
    if (crt) {
      st.crt_a = crt_exp_a(ld);
      DMB_LAUNCH(c, k_oz_res_a, dim3(blocks_for(Kh / 16, 128), (unsigned)Mpad), 128, 0, N, Kh, Mpad,
                 c->d_Z.as<float2>(), st.rs.as<double>(), std::ldexp(1.0, st.crt_a), oz_mods(OZ_NMOD),
                 st.A.as<signed char>());
    } else {
      DMB_LAUNCH(c, k_oz_slice_a, dim3(blocks_for(Kh, 256), (unsigned)Mpad), 256, 0, N, Kh, Mpad,
                 c->d_Z.as<float2>(), st.rs.as<double>(), st.A.as<signed char>());
    }
    make_map_bytes(&st.mapA, st.A.p, CU_TENSOR_MAP_DATA_TYPE_UINT8, (uint64_t)ld, (uint64_t)ld,
                   (uint64_t)(planes * 2 * Mpad), OZ_BK, OZ_BM);
    st.a_version = c->z_version;
    st.a_n = N;
    st.a_scheme = c->int8_scheme;
  }
}

void oz_zx(dmb_ctx *c, const double2 *X, double2 *Y, int64_t R, int lmax) {
  DMB_REQUIRE(lmax >= 0 && lmax <= OZ_LMAX, DMB_ERR_ARGUMENT, "int8 slice levels out of range");
  oz_prepare(c);
  OzState &st = oz_state(c);
  const int64_t N = c->n, Kh = round_up(N, OZ_BK), Mpad = round_up(N, 128), Rpad = round_up(R, OZ_BN);
  const int64_t ld = 2 * Kh;
  const bool crt = c->int8_scheme == 0;
  const int planes = crt ? OZ_NMOD : OZ_S;
  st.cs.ensure(sizeof(double) * Rpad);
  st.B.ensure((size_t)planes * Rpad * ld);
  if (st.b_key != Rpad || st.b_n != N || st.b_scheme != c->int8_scheme) {
    make_map_bytes(&st.mapB, st.B.p, CU_TENSOR_MAP_DATA_TYPE_UINT8, (uint64_t)ld, (uint64_t)ld,
                   (uint64_t)(planes * Rpad), OZ_BK, OZ_BN);
    make_map_bytes(&st.mapB128, st.B.p, CU_TENSOR_MAP_DATA_TYPE_UINT8, (uint64_t)ld, (uint64_t)ld,
                   (uint64_t)(planes * Rpad), OZ_BK, 128);
    st.b_key = Rpad;
    st.b_n = N;
    st.b_scheme = c->int8_scheme;
  }
  DMB_LAUNCH(c, k_oz_col_scale, (unsigned)R, 256, 0, N, X, st.cs.as<double>());
  OzSched sc{};
  int n = 0;
  if (crt) {
    // one product per modulus: 13 for the residuals, 12 for the Krylov
    // operator (the Z planes are shared; X gets the bits the moduli allow)
    const int nm = lmax >= OZ_LEVELS_RESIDUAL ? OZ_NMOD : OZ_NMOD - 1;
    const CrtConst k = crt_const(nm);
    const int b = crt_exp_b(ld, st.crt_a, k);
    DMB_REQUIRE(b >= 24, DMB_ERR_STATE, "int8 residue product: too few bits left for X");
    DMB_LAUNCH(c, k_oz_res_b, dim3(blocks_for(Kh / 16, 128), (unsigned)Rpad), 128, 0, N, R, Kh, Rpad, X,
               st.cs.as<double>(), std::ldexp(1.0, b), oz_mods(nm), st.B.as<signed char>());
    for (int i = 0; i < nm; i++, n++) {
      sc.arow[n] = (int)(i * 2 * Mpad);
      sc.brow[n] = (int)(i * Rpad);
      sc.close[n] = 1;
      sc.lscale[n] = 0.0;
      sc.mod[n] = OZ_MODULI[i];
      sc.mmul[n] = (unsigned)((((uint64_t)1 << 39) + OZ_MODULI[i] - 1) / OZ_MODULI[i]);
      sc.moff[n] = (unsigned)(OZ_MODULI[i] * ((1u << 31) / OZ_MODULI[i]));
      sc.frac[n] = k.frac[i];
      sc.fraclo[n] = k.fraclo[i];
    }
    sc.cscale = std::ldexp((double)k.M, -64 - st.crt_a - b);
  } else {
    DMB_LAUNCH(c, k_oz_slice_b, dim3(blocks_for(Kh, 256), (unsigned)Rpad), 256, 0, N, R, Kh, Rpad, X,
               st.cs.as<double>(), st.B.as<signed char>());
    // pair schedule: levels L = p + q <= lmax, largest terms first; a level's
    // pairs share one TMEM sum unless int32 headroom forces an earlier drain
    const int64_t maxp = (int64_t)(2147483647.0 / (16129.0 * (double)ld));
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
  }
  sc.n = n;
  // persistent grid: data-parallel full waves, stream-K tail (k_oz_gemm)
  const int ncol = (int)(Rpad / OZ_BN);
  const int64_t ntiles = (round_up(N, 64) / 64) * ncol;
  const int64_t G = std::min<int64_t>(ntiles, std::max(1, c->sm_count));
  const int64_t F = (ntiles / G) * G, Wt = (ntiles - F) * n;
  if (crt) {
    // tile shape from the autotuner, per (row tiles, column tiles): one-SM
    // 64 x 256 complex tiles (k_oz_gemm) or CTA-pair 128 x 256 tiles
    // (k_oz_pair); both give the same bits (integer sums)
    const int64_t tb1 = dmb::tune_bucket(Mpad / 128), tb2 = ncol;
    const int cand = dmb::tune_choose(c, dmb::TUNE_OZ_TILE, tb1, tb2, 2);
    dmb::TuneMark mk;
    if (cand == 1) {
      // residue planes: as below, per CTA of the pairs and per half of a
      // tail pair tile
      const int64_t npairs = (Mpad / 128) * ncol;
      const int64_t G2 = std::min<int64_t>(npairs, std::max(1, c->sm_count / 2));
      const int64_t F2 = (npairs / G2) * G2;
      st.Rres.ensure((size_t)(2 * G2 + 2 * (npairs - F2)) * OZ_RES_TILE);
      if (!st.pair_attr) {
        DMB_CUDA(cudaFuncSetAttribute(k_oz_pair, cudaFuncAttributeMaxDynamicSharedMemorySize, OZP_SMEM));
        st.pair_attr = true;
      }
      kt_begin(c);
      dmb::tune_begin(c, dmb::TUNE_OZ_TILE, tb1, tb2, cand, mk);
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)(2 * G2));
      cfg.blockDim = dim3(320);
      cfg.dynamicSmemBytes = OZP_SMEM;
      cfg.stream = c->stream;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = 2;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      DMB_CUDA(cudaLaunchKernelEx(&cfg, k_oz_pair, st.mapA, st.mapB128, sc, (int)(ld / OZ_BK), (int64_t)N,
                                  (int64_t)R, Y, (int64_t)N, ncol, npairs, (const double *)st.rs.as<double>(),
                                  (const double *)st.cs.as<double>(), st.Rres.as<unsigned char>(),
                                  st.err.as<unsigned>()));
      c->launches++;
      dmb::tune_end(c, mk);
      if (npairs > F2)
        DMB_LAUNCH(c, k_oz_crt_tail, (unsigned)(2 * (npairs - F2)), 256, 0, sc, ncol, N, R, F2, (int)(2 * G2), 1, Y,
                   N, st.rs.as<double>(), st.cs.as<double>(), st.Rres.as<unsigned char>());
    } else {
      // residue planes: one tile's worth per CTA (its whole tiles, one at a
      // time) and one per tail tile (its moduli drained by several CTAs,
      // converted by k_oz_crt_tail)
      st.Rres.ensure((size_t)(G + ntiles - F) * OZ_RES_TILE);
      kt_begin(c);
      dmb::tune_begin(c, dmb::TUNE_OZ_TILE, tb1, tb2, cand, mk);
      DMB_LAUNCH(c, k_oz_gemm<true>, (unsigned)G, oz_threads<true>(), OZ_SMEM, st.mapA, st.mapB, sc,
                 (int)(ld / OZ_BK), N, R, Y, Y, N, ncol, ntiles, st.rs.as<double>(), st.cs.as<double>(),
                 st.Rres.as<unsigned char>(), st.err.as<unsigned>());
      dmb::tune_end(c, mk);
      if (ntiles > F)
        DMB_LAUNCH(c, k_oz_crt_tail, (unsigned)(ntiles - F), 256, 0, sc, ncol, N, R, F, (int)G, 0, Y, N,
                   st.rs.as<double>(), st.cs.as<double>(), st.Rres.as<unsigned char>());
    }
  } else {
    // the host replays the tail split to list each partial tile's slots
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
      st.fix.ensure(sizeof(int64_t) * fix.size());
      st.runs.ensure(sizeof(int) * runs.size());
      DMB_CUDA(cudaMemcpyAsync(st.fix.p, fix.data(), sizeof(int64_t) * fix.size(), cudaMemcpyHostToDevice,
                               c->stream));
      DMB_CUDA(cudaMemcpyAsync(st.runs.p, runs.data(), sizeof(int) * runs.size(), cudaMemcpyHostToDevice,
                               c->stream));
      st.P.ensure(sizeof(double2) * G * 2 * OZ_TILE_ELEMS);
    }
    kt_begin(c);
    double2 *Pw = fix.empty() ? Y : st.P.as<double2>();
    DMB_LAUNCH(c, k_oz_gemm<false>, (unsigned)G, oz_threads<false>(), OZ_SMEM, st.mapA, st.mapB, sc,
               (int)(ld / OZ_BK), N, R, Y, Pw, N, ncol, ntiles, st.rs.as<double>(), st.cs.as<double>(),
               (unsigned char *)nullptr, st.err.as<unsigned>());
    if (!runs.empty())
      DMB_LAUNCH(c, k_oz_fixup, (unsigned)runs.size(), 256, 0, st.fix.as<int64_t>(), st.runs.as<int>(), ncol, N, R,
                 Y, st.P.as<double2>(), N);
  }
  // int8 work: every product is a real (2N x 2N) x (2N x R) product
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
    for (DevBuf *b : {&st->A, &st->B, &st->rs, &st->cs, &st->err, &st->P, &st->fix, &st->runs, &st->Rres}) b->release();
    delete st;
    g_oz_states.erase(g_oz_states.begin() + i);
    return;
  }
}

}  // namespace dmb
