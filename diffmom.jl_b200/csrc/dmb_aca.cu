// dmb_aca.cu -- H-matrix EFIE operator by adaptive cross approximation.
//
// Reference path: build_aca_operator (src/fast/ACA.jl:802-1103), the path of
// solve_scattering for 10k < N <= 50k (src/Workflow.jl:204-210).
//
//   host     cluster tree by median bisection of the RWG centres
//            (src/fast/ClusterTree.jl:82-166) and the block tasks of
//            _enum_block_tasks! (src/fast/ACA.jl:696-738) with is_admissible
//            (src/fast/ClusterTree.jl:223-246).  Integer bookkeeping.
//   device   one kernel fills every dense block with FP64 EFIE entries; one
//            CTA per admissible block runs the partially pivoted ACA of
//            aca_lowrank (src/fast/ACA.jl:351-554), all blocks at once.  An
//            entry is evaluated on the fly with the same arithmetic as the
//            dense assembly: the far triangle-pair value of its four slot
//            pairs plus the precomputed singular records of near pairs.
//   product  y = A x as four launches per right-hand side: gather x into tree
//            order; t_b = V_b^H x_b for every low-rank block; the partial
//            product of every block (D_b x_b or U_b t_b, one CTA per block);
//            per leaf, the partials of the blocks covering it summed and
//            scattered to the original order.  Fixed summation order, no
//            atomics; the adjoint and the transpose use the column side.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <numeric>
#include <type_traits>

#include "dmb_device.cuh"
#include "dmb_internal.h"

namespace {

unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// ---------------------------------------------------------------------------
// exact admissibility near the decision boundary
// ---------------------------------------------------------------------------
// Nonnegative big integer (little-endian 32-bit limbs) with the few operations
// the comparison min(diam)^2 <= eta^2 dist^2 needs on values that are exact
// differences of doubles.
struct BigInt {
  bool neg = false;
  std::vector<uint32_t> d;
};

void big_trim(std::vector<uint32_t> &d) {
  while (!d.empty() && d.back() == 0) d.pop_back();
}

int mag_cmp(const std::vector<uint32_t> &a, const std::vector<uint32_t> &b) {
  if (a.size() != b.size()) return a.size() < b.size() ? -1 : 1;
  for (size_t i = a.size(); i-- > 0;)
    if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
  return 0;
}

std::vector<uint32_t> mag_add(const std::vector<uint32_t> &a, const std::vector<uint32_t> &b) {
  std::vector<uint32_t> r(std::max(a.size(), b.size()) + 1, 0);
  uint64_t carry = 0;
  for (size_t i = 0; i < r.size(); i++) {
    uint64_t s = carry + (i < a.size() ? a[i] : 0) + (i < b.size() ? b[i] : 0);
    r[i] = (uint32_t)s;
    carry = s >> 32;
  }
  big_trim(r);
  return r;
}

// a - b for |a| >= |b|
std::vector<uint32_t> mag_sub(const std::vector<uint32_t> &a, const std::vector<uint32_t> &b) {
  std::vector<uint32_t> r(a.size(), 0);
  int64_t borrow = 0;
  for (size_t i = 0; i < a.size(); i++) {
    int64_t s = (int64_t)a[i] - borrow - (i < b.size() ? (int64_t)b[i] : 0);
    borrow = s < 0;
    if (s < 0) s += (int64_t)1 << 32;
    r[i] = (uint32_t)s;
  }
  big_trim(r);
  return r;
}

std::vector<uint32_t> mag_mul(const std::vector<uint32_t> &a, const std::vector<uint32_t> &b) {
  if (a.empty() || b.empty()) return {};
  std::vector<uint64_t> acc(a.size() + b.size() + 1, 0);
  for (size_t i = 0; i < a.size(); i++) {
    uint64_t carry = 0;
    for (size_t j = 0; j < b.size(); j++) {
      uint64_t cur = acc[i + j] + (uint64_t)a[i] * b[j] + carry;
      acc[i + j] = cur & 0xffffffffu;
      carry = cur >> 32;
    }
    size_t k = i + b.size();
    while (carry) {
      uint64_t cur = acc[k] + carry;
      acc[k] = cur & 0xffffffffu;
      carry = cur >> 32;
      k++;
    }
  }
  std::vector<uint32_t> r(acc.size());
  for (size_t i = 0; i < acc.size(); i++) r[i] = (uint32_t)acc[i];
  big_trim(r);
  return r;
}

std::vector<uint32_t> mag_shl(const std::vector<uint32_t> &a, int64_t bits) {
  if (a.empty()) return {};
  const int64_t w = bits / 32, s = bits % 32;
  std::vector<uint32_t> r((size_t)w + a.size() + 1, 0);
  for (size_t i = 0; i < a.size(); i++) {
    uint64_t v = (uint64_t)a[i] << s;
    r[w + i] |= (uint32_t)v;
    r[w + i + 1] |= (uint32_t)(v >> 32);
  }
  big_trim(r);
  return r;
}

BigInt big_sub(const BigInt &a, const BigInt &b) {
  BigInt r;
  if (a.neg != b.neg) {  // a - b = a + (-b)
    r.d = mag_add(a.d, b.d);
    r.neg = a.neg;
  } else if (mag_cmp(a.d, b.d) >= 0) {
    r.d = mag_sub(a.d, b.d);
    r.neg = a.neg;
  } else {
    r.d = mag_sub(b.d, a.d);
    r.neg = !a.neg;
  }
  if (r.d.empty()) r.neg = false;
  return r;
}

int big_cmp(const BigInt &a, const BigInt &b) {
  if (a.neg != b.neg) return a.neg ? -1 : 1;
  int c = mag_cmp(a.d, b.d);
  return a.neg ? -c : c;
}

const BigInt &big_max(const BigInt &a, const BigInt &b) { return big_cmp(a, b) >= 0 ? a : b; }
const BigInt &big_min(const BigInt &a, const BigInt &b) { return big_cmp(a, b) <= 0 ? a : b; }

// x = m * 2^e with an integer 53-bit m
void split_double(double x, uint64_t &m, int &e) {
  if (x == 0.0) {
    m = 0;
    e = 0;
    return;
  }
  int ex = 0;
  double f = std::frexp(std::fabs(x), &ex);
  m = (uint64_t)std::ldexp(f, 53);
  e = ex - 53;
}

// _cluster_admissibility_exact (src/fast/ClusterTree.jl:193-214):
// min(max span_i, max span_j)^2 <= eta^2 |gap|^2 in exact rationals
bool admissible_exact(const double *bi_min, const double *bi_max, const double *bj_min, const double *bj_max,
                      double eta) {
  const double *src[4] = {bi_min, bi_max, bj_min, bj_max};
  uint64_t mm[12];
  int ee[12];
  int e0 = 0;
  bool any = false;
  for (int a = 0; a < 4; a++)
    for (int c = 0; c < 3; c++) {
      split_double(src[a][c], mm[3 * a + c], ee[3 * a + c]);
      if (mm[3 * a + c] != 0) {
        e0 = any ? std::min(e0, ee[3 * a + c]) : ee[3 * a + c];
        any = true;
      }
    }
  BigInt v[12];
  for (int i = 0; i < 12; i++) {
    if (mm[i] == 0) continue;
    std::vector<uint32_t> base = {(uint32_t)mm[i], (uint32_t)(mm[i] >> 32)};
    big_trim(base);
    v[i].d = mag_shl(base, ee[i] - e0);
    v[i].neg = src[i / 3][i % 3] < 0;
  }
  const BigInt *imin = v, *imax = v + 3, *jmin = v + 6, *jmax = v + 9;
  BigInt zero;
  std::vector<uint32_t> dist2;
  BigInt span_i, span_j;
  for (int c = 0; c < 3; c++) {
    BigInt g1 = big_sub(imin[c], jmax[c]), g2 = big_sub(jmin[c], imax[c]);
    const BigInt &g = big_max(big_max(g1, g2), zero);
    dist2 = mag_add(dist2, mag_mul(g.d, g.d));
    BigInt si = big_sub(imax[c], imin[c]), sj = big_sub(jmax[c], jmin[c]);
    span_i = c == 0 ? si : big_max(span_i, si);
    span_j = c == 0 ? sj : big_max(span_j, sj);
  }
  const BigInt &diam = big_min(span_i, span_j);
  std::vector<uint32_t> lhs = mag_mul(diam.d, diam.d);
  uint64_t me;
  int ex;
  split_double(eta, me, ex);
  std::vector<uint32_t> em = {(uint32_t)me, (uint32_t)(me >> 32)};
  big_trim(em);
  std::vector<uint32_t> rhs = mag_mul(mag_mul(em, em), dist2);
  if (ex >= 0)
    rhs = mag_shl(rhs, 2 * (int64_t)ex);
  else
    lhs = mag_shl(lhs, -2 * (int64_t)ex);
  return mag_cmp(lhs, rhs) <= 0;
}

// eps(x) of Julia: distance from |x| to the next larger double
double ulp_above(double x) {
  x = std::fabs(x);
  return std::nextafter(x, INFINITY) - x;
}

double box_diameter(const double *bmin, const double *bmax) {
  double s0 = bmax[0] - bmin[0], s1 = bmax[1] - bmin[1], s2 = bmax[2] - bmin[2];
  DMB_REQUIRE(std::isfinite(s0) && std::isfinite(s1) && std::isfinite(s2) && s0 >= 0 && s1 >= 0 && s2 >= 0,
              DMB_ERR_ARGUMENT, "cluster has invalid bounding-box extents");
  return std::max(s0, std::max(s1, s2));
}

// is_admissible (src/fast/ClusterTree.jl:223-246): floating-point decision
// outside a 64-ulp band around the boundary, exact rational one inside it
bool box_admissible(const double *bi_min, const double *bi_max, const double *bj_min, const double *bj_max,
                    double eta) {
  DMB_REQUIRE(std::isfinite(eta) && eta > 0.0, DMB_ERR_ARGUMENT,
              "eta must be finite and positive, got " + std::to_string(eta));
  double g[3];
  for (int c = 0; c < 3; c++) {
    g[c] = std::max(std::max(bi_min[c] - bj_max[c], bj_min[c] - bi_max[c]), 0.0);
    DMB_REQUIRE(std::isfinite(g[c]), DMB_ERR_OVERFLOW, "cluster bounding-box separation is non-finite");
  }
  double d = std::sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
  if ((d == 0.0 || !std::isfinite(d)) && (g[0] != 0 || g[1] != 0 || g[2] != 0)) {
    const double s = std::max(g[0], std::max(g[1], g[2]));  // underflow / overflow of the squares
    d = s * std::sqrt((g[0] / s) * (g[0] / s) + (g[1] / s) * (g[1] / s) + (g[2] / s) * (g[2] / s));
  }
  DMB_REQUIRE(std::isfinite(d), DMB_ERR_OVERFLOW, "cluster distance overflowed");
  if (d <= 0.0) return false;  // overlapping or touching
  const double diam = std::min(box_diameter(bi_min, bi_max), box_diameter(bj_min, bj_max));
  const double sd = eta * d;
  if (std::isinf(sd)) return true;
  if (sd == 0.0) return diam == 0.0;
  const double unc = 64 * ulp_above(std::max(diam, sd));
  if (std::isfinite(unc) && std::fabs(diam - sd) > unc) return diam <= sd;
  return admissible_exact(bi_min, bi_max, bj_min, bj_max, eta);
}

// ---------------------------------------------------------------------------
// cluster tree and block tasks
// ---------------------------------------------------------------------------
struct Node {
  int64_t lo, hi;  // tree-order positions, inclusive, 0-based
  double bmin[3], bmax[3];
  int64_t left = -1, right = -1;
  int level = 0;
};
struct Task {
  int64_t row, col;
  int kind;  // 0 dense, 1 low-rank
};
struct Plan {
  std::vector<Node> nodes;
  std::vector<int64_t> perm;
  std::vector<Task> tasks;
};

// isless of Julia on finite doubles (-0.0 before 0.0)
bool jl_isless(double a, double b) { return a < b || (a == b && std::signbit(a) && !std::signbit(b)); }

void build_tree(const double *ctr, int64_t n, int leaf_size, Plan &P) {
  DMB_REQUIRE(n > 0, DMB_ERR_ARGUMENT, "build_cluster_tree: centers must not be empty");
  DMB_REQUIRE(leaf_size >= 1, DMB_ERR_ARGUMENT,
              "build_cluster_tree: leaf_size must be at least 1, got " + std::to_string(leaf_size));
  // _cluster_tree_resource_bounds (src/fast/ClusterTree.jl:13-36) with the
  // default limits (30,000,000 nodes, 2e9 bytes of 88-byte nodes + 3 index vectors)
  int64_t target = (n + leaf_size - 1) / leaf_size, leaves = 1;
  while (leaves < target) leaves *= 2;
  const int64_t node_bound = 2 * leaves - 1;
  DMB_REQUIRE(node_bound <= 30000000, DMB_ERR_ARGUMENT,
              "cluster tree requires at most " + std::to_string(node_bound) +
                  " nodes, exceeding max_nodes=30000000");
  const double storage = (double)node_bound * 88.0 + 24.0 * (double)n;
  DMB_REQUIRE(storage <= 2e9, DMB_ERR_ARGUMENT,
              "cluster-tree arrays require " + std::to_string((int64_t)storage) +
                  " bytes, exceeding max_storage_bytes=2000000000");
  for (int64_t i = 0; i < n; i++)
    for (int c = 0; c < 3; c++)
      DMB_REQUIRE(std::isfinite(ctr[3 * i + c]), DMB_ERR_ARGUMENT,
                  "build_cluster_tree: center " + std::to_string(i + 1) + " must be finite");
  P.perm.resize(n);
  std::iota(P.perm.begin(), P.perm.end(), (int64_t)0);
  P.nodes.clear();
  P.nodes.reserve((size_t)std::min<int64_t>(node_bound, 4 * target + 8));
  // preorder: a node, then its left and right subtrees (depth ~ log2(n / leaf_size))
  std::function<int64_t(int64_t, int64_t, int)> build = [&](int64_t lo, int64_t hi, int level) -> int64_t {
    Node nd;
    nd.lo = lo;
    nd.hi = hi;
    nd.level = level;
    for (int c = 0; c < 3; c++) {
      nd.bmin[c] = INFINITY;
      nd.bmax[c] = -INFINITY;
    }
    for (int64_t k = lo; k <= hi; k++)
      for (int c = 0; c < 3; c++) {
        const double v = ctr[3 * P.perm[k] + c];
        nd.bmin[c] = std::min(nd.bmin[c], v);
        nd.bmax[c] = std::max(nd.bmax[c], v);
      }
    double span[3];
    for (int c = 0; c < 3; c++) {
      span[c] = nd.bmax[c] - nd.bmin[c];
      DMB_REQUIRE(std::isfinite(span[c]), DMB_ERR_ARGUMENT,
                  "build_cluster_tree: cluster coordinate extent is too large");
    }
    if (hi - lo + 1 <= leaf_size) {
      P.nodes.push_back(nd);
      return (int64_t)P.nodes.size() - 1;
    }
    int axis = 0;
    if (span[1] > span[axis]) axis = 1;
    if (span[2] > span[axis]) axis = 2;
    std::stable_sort(P.perm.begin() + lo, P.perm.begin() + hi + 1,
                     [&](int64_t a, int64_t b) { return jl_isless(ctr[3 * a + axis], ctr[3 * b + axis]); });
    // mid = (lo + hi) >> 1 on the reference's 1-based positions
    const int64_t mid = ((lo + 1 + hi + 1) >> 1) - 1;
    P.nodes.push_back(nd);
    const int64_t me = (int64_t)P.nodes.size() - 1;
    const int64_t l = build(lo, mid, level + 1);
    const int64_t r = build(mid + 1, hi, level + 1);
    P.nodes[me].left = l;
    P.nodes[me].right = r;
    return me;
  };
  build(0, n - 1, 0);
}

bool node_admissible(const Plan &P, int64_t i, int64_t j, double eta) {
  const Node &a = P.nodes[i], &b = P.nodes[j];
  return box_admissible(a.bmin, a.bmax, b.bmin, b.bmax, eta);
}

void enum_tasks(Plan &P, int64_t rn, int64_t cn, double eta, int64_t max_tasks) {
  DMB_REQUIRE((int64_t)P.tasks.size() < max_tasks, DMB_ERR_ARGUMENT,
              "ACA block enumeration exceeds max_block_tasks=" + std::to_string(max_tasks));
  if (node_admissible(P, rn, cn, eta)) {
    P.tasks.push_back({rn, cn, 1});
    return;
  }
  const Node &r = P.nodes[rn], &c = P.nodes[cn];
  const bool rl = r.left < 0, cl = c.left < 0;
  if (rl && cl) {
    P.tasks.push_back({rn, cn, 0});
    return;
  }
  const int64_t r_left = r.left, r_right = r.right, c_left = c.left, c_right = c.right;
  if (rl) {
    enum_tasks(P, rn, c_left, eta, max_tasks);
    enum_tasks(P, rn, c_right, eta, max_tasks);
  } else if (cl) {
    enum_tasks(P, r_left, cn, eta, max_tasks);
    enum_tasks(P, r_right, cn, eta, max_tasks);
  } else {
    enum_tasks(P, r_left, c_left, eta, max_tasks);
    enum_tasks(P, r_left, c_right, eta, max_tasks);
    enum_tasks(P, r_right, c_left, eta, max_tasks);
    enum_tasks(P, r_right, c_right, eta, max_tasks);
  }
}

void make_plan(const double *ctr, int64_t n, int leaf_size, double eta, int64_t max_tasks, Plan &P) {
  DMB_REQUIRE(leaf_size >= 1, DMB_ERR_ARGUMENT, "ACA leaf_size must be at least 1, got " + std::to_string(leaf_size));
  DMB_REQUIRE(std::isfinite(eta) && eta > 0.0, DMB_ERR_ARGUMENT,
              "ACA eta must be finite and positive, got " + std::to_string(eta));
  DMB_REQUIRE(max_tasks >= 1, DMB_ERR_ARGUMENT,
              "max_block_tasks must be positive, got " + std::to_string(max_tasks));
  build_tree(ctr, n, leaf_size, P);
  P.tasks.clear();
  enum_tasks(P, 0, 0, eta, max_tasks);
}

// ---------------------------------------------------------------------------
// device: EFIE entries on the fly
// ---------------------------------------------------------------------------
struct AcaGeo {
  const TriCache *tc;
  const int *rslot;
  const int *aoff, *anb;
  const int2 *near_mn;
  const int64_t *near_off;
  const double2 *near_val;
  int64_t n_near;
  double k, inv_k2, omega_mu0;
};

__device__ __forceinline__ bool aca_tri_adjacent(const int *__restrict__ off, const int *__restrict__ nb, int ta,
                                                 int tb) {
  for (int i = off[ta]; i < off[ta + 1]; i++)
    if (nb[i] == tb) return true;
  return false;
}

// Element (i, j) of the far triangle-pair block of (A, B), A the triangle of
// the lower slot index: the moments and the contraction are written as in the
// dense assembly's far-pair kernel, so both give the same value.
template <int NQ>
__device__ double2 far_slot_value(const TriCache &A, const TriCache &B, int i, int j, double k, double inv_k2) {
  double m0r = 0, m0i = 0, mar[3] = {0, 0, 0}, mai[3] = {0, 0, 0}, mbr[3] = {0, 0, 0}, mbi[3] = {0, 0, 0},
         mabr = 0, mabi = 0;
  // same operations in the same order; the points of A are read where they
  // are used (cached) instead of held in registers
#pragma unroll 1
  for (int b = 0; b < NQ; b++) {
    const double qb0 = B.qp[b][0], qb1 = B.qp[b][1], qb2 = B.qp[b][2];
    const double lb0 = B.ql[b][0], lb1 = B.ql[b][1], lb2 = B.ql[b][2];
    const double wb = B.w2a[b];
#pragma unroll 1
    for (int a = 0; a < NQ; a++) {
      const double la0 = A.ql[a][0], la1 = A.ql[a][1], la2 = A.ql[a][2];
      double dx = A.qp[a][0] - qb0, dy = A.qp[a][1] - qb1, dz = A.qp[a][2] - qb2;
      double R = sqrt(dx * dx + dy * dy + dz * dz);
      double sn, cs;
      sincos(k * R, &sn, &cs);
      double g = (DMB_INV_FOUR_PI / R) * (A.w2a[a] * wb);
      double gr = cs * g, gi = -sn * g;
      m0r += gr;
      m0i += gi;
      mar[0] = fma(gr, la0, mar[0]); mai[0] = fma(gi, la0, mai[0]);
      mar[1] = fma(gr, la1, mar[1]); mai[1] = fma(gi, la1, mai[1]);
      mar[2] = fma(gr, la2, mar[2]); mai[2] = fma(gi, la2, mai[2]);
      mbr[0] = fma(gr, lb0, mbr[0]); mbi[0] = fma(gi, lb0, mbi[0]);
      mbr[1] = fma(gr, lb1, mbr[1]); mbi[1] = fma(gi, lb1, mbi[1]);
      mbr[2] = fma(gr, lb2, mbr[2]); mbi[2] = fma(gi, lb2, mbi[2]);
      double dd = la0 * lb0 + la1 * lb1 + la2 * lb2;
      mabr = fma(gr, dd, mabr);
      mabi = fma(gi, dd, mabi);
    }
  }
  double si = A.s[i], dvi = A.dv[i];
  double pi0 = A.pl[i][0], pi1 = A.pl[i][1], pi2 = A.pl[i][2];
  double mbpr = mbr[0] * pi0 + mbr[1] * pi1 + mbr[2] * pi2;
  double mbpi = mbi[0] * pi0 + mbi[1] * pi1 + mbi[2] * pi2;
  double sj = B.s[j], dvj = B.dv[j];
  double pj0 = B.pl[j][0], pj1 = B.pl[j][1], pj2 = B.pl[j][2];
  double mapr = mar[0] * pj0 + mar[1] * pj1 + mar[2] * pj2;
  double mapi = mai[0] * pj0 + mai[1] * pj1 + mai[2] * pj2;
  double pp = pi0 * pj0 + pi1 * pj1 + pi2 * pj2;
  double ss = si * sj, sc = dvi * dvj * inv_k2;
  double vr = ss * (mabr - mapr - mbpr + pp * m0r) - sc * m0r;
  double vi = ss * (mabi - mapi - mbpi + pp * m0i) - sc * m0i;
  return make_double2(vr, vi);
}

// Z[m][n] (0-based) in the dense assembly's order of operations: the four
// slot-pair values summed (a over m's slots, b over n's), times -i omega mu0,
// plus the entry's near records summed in their fixed order
template <int NQ>
__device__ double2 aca_entry(const AcaGeo &g, int m, int n) {
  const int sm[2] = {g.rslot[2 * m], g.rslot[2 * m + 1]};
  const int sn[2] = {g.rslot[2 * n], g.rslot[2 * n + 1]};
  double re = 0, im = 0;
  bool near = false;
  // the four slot pairs one after another (unrolled, their quadrature loops
  // would hold four sets of moments in registers)
#pragma unroll 1
  for (int a = 0; a < 2; a++)
#pragma unroll 1
    for (int b = 0; b < 2; b++) {
      const int x = sm[a], y = sn[b];
      const int lo = x <= y ? x : y, hi = x <= y ? y : x;
      const int ta = lo / 3, tb = hi / 3;
      double2 v = make_double2(0.0, 0.0);
      if (ta == tb || aca_tri_adjacent(g.aoff, g.anb, ta, tb))
        near = true;
      else
        v = far_slot_value<NQ>(g.tc[ta], g.tc[tb], lo - 3 * ta, hi - 3 * tb, g.k, g.inv_k2);
      re += v.x;
      im += v.y;
    }
  double2 z = make_double2(g.omega_mu0 * im, -g.omega_mu0 * re);
  if (near && g.n_near > 0) {
    const int a = m <= n ? m : n, b = m <= n ? n : m;
    int64_t lo = 0, hi = g.n_near;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      const int2 e = g.near_mn[mid];
      if (e.x < a || (e.x == a && e.y < b))
        lo = mid + 1;
      else
        hi = mid;
    }
    if (lo < g.n_near && g.near_mn[lo].x == a && g.near_mn[lo].y == b) {
      double nr = 0, ni = 0;
      for (int64_t r = g.near_off[lo]; r < g.near_off[lo + 1]; r++) {
        nr += g.near_val[r].x;
        ni += g.near_val[r].y;
      }
      z = cadd(z, make_double2(g.omega_mu0 * ni, -g.omega_mu0 * nr));
    }
  }
  return z;
}

// ---------------------------------------------------------------------------
// device: block fill and ACA
// ---------------------------------------------------------------------------
template <int NQ>
__global__ void __launch_bounds__(256) k_aca_dense(AcaGeo g, const AcaBlockDesc *__restrict__ blocks,
                                                   const int *__restrict__ ids, const int *__restrict__ perm,
                                                   double2 *__restrict__ arena) {
  const AcaBlockDesc bd = blocks[ids[blockIdx.x]];
  double2 *D = arena + bd.off_a;
  const int64_t cnt = (int64_t)bd.m * bd.n;
  for (int64_t e = threadIdx.x; e < cnt; e += blockDim.x) {
    const int ii = (int)(e % bd.m), jj = (int)(e / bd.m);
    D[e] = aca_entry<NQ>(g, perm[bd.r0 + ii], perm[bd.c0 + jj]);
  }
}

__global__ void k_aca_entries(AcaGeo g, int nq, int64_t count, const int *__restrict__ mn, double2 *__restrict__ out) {
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count) return;
  const int m = mn[2 * e], n = mn[2 * e + 1];
  double2 v;
  if (nq == 1) v = aca_entry<1>(g, m, n);
  else if (nq == 3) v = aca_entry<3>(g, m, n);
  else if (nq == 4) v = aca_entry<4>(g, m, n);
  else v = aca_entry<7>(g, m, n);
  out[e] = v;
}

// scaled magnitude (fraction in [0.5, 1), binary exponent) of
// src/fast/ACA.jl:232-306
struct Mag {
  double f;
  int e;
};
__device__ __forceinline__ Mag mag_make(double x) {
  Mag r;
  r.f = frexp(x, &r.e);
  return r;
}
__device__ __forceinline__ Mag mag_mul(Mag a, Mag b) {
  Mag r;
  r.f = frexp(a.f * b.f, &r.e);
  r.e += a.e + b.e;
  return r;
}
__device__ __forceinline__ bool mag_less(Mag a, Mag b) { return a.e == b.e ? a.f < b.f : a.e < b.e; }
__device__ __forceinline__ double mag_ratio(Mag a, Mag b) { return ldexp(a.f / b.f, a.e - b.e); }

// (value, index) arg-max over the CTA: larger value wins, ties go to the
// smaller index (the reference scans in order with a strict comparison)
__device__ void block_argmax(double &v, int &idx, double *sv, int *si) {
  for (int o = 16; o > 0; o >>= 1) {
    double ov = __shfl_xor_sync(0xffffffffu, v, o);
    int oi = __shfl_xor_sync(0xffffffffu, idx, o);
    if (ov > v || (ov == v && oi >= 0 && (idx < 0 || oi < idx))) {
      v = ov;
      idx = oi;
    }
  }
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    sv[w] = v;
    si[w] = idx;
  }
  __syncthreads();
  v = sv[0];
  idx = si[0];
  for (int q = 1; q < nw; q++)
    if (sv[q] > v || (sv[q] == v && si[q] >= 0 && (idx < 0 || si[q] < idx))) {
      v = sv[q];
      idx = si[q];
    }
}

// three maxima (sh: 96 doubles) and two sums (sh: 64 doubles) with one barrier pair
__device__ void block_max3(double &a, double &b, double &c, double *sh) {
  a = warp_max(a);
  b = warp_max(b);
  c = warp_max(c);
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    sh[w] = a;
    sh[32 + w] = b;
    sh[64 + w] = c;
  }
  __syncthreads();
  a = sh[0];
  b = sh[32];
  c = sh[64];
  for (int q = 1; q < nw; q++) {
    a = fmax(a, sh[q]);
    b = fmax(b, sh[32 + q]);
    c = fmax(c, sh[64 + q]);
  }
}
__device__ void block_sum2(double &a, double &b, double *sh) {
  a = warp_sum(a);
  b = warp_sum(b);
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    sh[w] = a;
    sh[32 + w] = b;
  }
  __syncthreads();
  a = 0;
  b = 0;
  for (int q = 0; q < nw; q++) {
    a += sh[q];
    b += sh[32 + q];
  }
}
__device__ double block_max(double v, double *sh) {
  v = warp_max(v);
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[w] = v;
  __syncthreads();
  double s = sh[0];
  for (int q = 1; q < nw; q++) s = fmax(s, sh[q]);
  return s;
}

// per-rank scratch of one low-rank block: 10 doubles per rank
constexpr int ACA_SCR = 10;  // su, nu, sv, nv, term f, term e, <U_p,u> re/im, <V_p,v> re/im

// One CTA per admissible block: aca_lowrank (src/fast/ACA.jl:351-554).
// status: 0 ok, 1 non-finite update (the block becomes dense), 2 zero-norm
// update; conv: 1 converged, 0 stopped otherwise.
// NT threads per CTA: the launcher buckets the blocks by size (small blocks
// on narrow CTAs, the few large ones on wide CTAs).
template <int NQ, int NT>
__global__ void __launch_bounds__(NT) k_aca_lowrank(AcaGeo g, const AcaBlockDesc *__restrict__ blocks,
                                                    const int *__restrict__ ids, const int *__restrict__ perm,
                                                    double2 *__restrict__ arena, const int64_t *__restrict__ foff,
                                                    unsigned char *__restrict__ flags,
                                                    const int64_t *__restrict__ soff, double *__restrict__ scr,
                                                    double tol, int *__restrict__ rank_out,
                                                    int *__restrict__ status_out, int *__restrict__ conv_out) {
  __shared__ double sv[32];
  __shared__ int si[32];
  __shared__ double sh[96];
  __shared__ int s_pc, s_stop, s_conv;
  __shared__ double2 s_pivot;
  const int bi = ids[blockIdx.x];
  const AcaBlockDesc bd = blocks[bi];
  const int m = bd.m, n = bd.n, rmax = bd.rmax;
  double2 *U = arena + bd.off_a, *V = arena + bd.off_b;
  unsigned char *urow = flags + foff[blockIdx.x], *ucol = urow + m;
  double *S = scr + soff[blockIdx.x];
  const int *rows = perm + bd.r0, *cols = perm + bd.c0;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  int prow = 0, rank = 0, status = 0;
  bool converged = false;
  // Frobenius estimate in units of the largest rank-one term (thread 0)
  Mag fscale{0.0, 0};
  double fsq = 0.0;
  for (int k = 0; k < rmax; k++) {
    double2 *Uk = U + (int64_t)k * m, *Vk = V + (int64_t)k * n;
    // residual row at prow -> Vk (not yet conjugated); arg-max over unused columns
    const int ri = rows[prow];
    double best = 0.0;
    int bidx = -1;
    for (int jj = tid; jj < n; jj += nt) {
      double2 v = aca_entry<NQ>(g, ri, cols[jj]);
      for (int p = 0; p < k; p++) {
        const double2 u = U[prow + (int64_t)p * m], w = V[jj + (int64_t)p * n];
        v = csub(v, cmul(u, cconj(w)));
      }
      Vk[jj] = v;
      const double av = hypot(v.x, v.y);
      if (av > best && !ucol[jj]) {
        best = av;
        bidx = jj;
      }
    }
    block_argmax(best, bidx, sv, si);
    if (tid == 0) {
      s_stop = 0;
      s_pc = bidx;
    }
    __syncthreads();
    if (bidx < 0 || best == 0.0) {
      // no positive pivot: the first unused column, if any and nonzero
      int first = n;
      for (int jj = tid; jj < n; jj += nt)
        if (!ucol[jj]) {
          first = jj;
          break;
        }
      double fv = (double)first;
      fv = -block_max(-fv, sh);
      if (tid == 0) {
        if ((int)fv >= n) {
          s_stop = 1;
        } else {
          const double2 v = Vk[(int)fv];
          s_pc = (int)fv;
          if (hypot(v.x, v.y) == 0.0) s_stop = 1;
        }
      }
      __syncthreads();
    }
    if (s_stop) break;
    const int pc = s_pc;
    if (tid == 0) s_pivot = Vk[pc];
    __syncthreads();
    const double2 piv = s_pivot;
    // residual column at pc -> Uk = col / pivot
    const int cj = cols[pc];
    for (int ii = tid; ii < m; ii += nt) {
      double2 u = aca_entry<NQ>(g, rows[ii], cj);
      for (int p = 0; p < k; p++) {
        const double2 a = U[ii + (int64_t)p * m], w = V[pc + (int64_t)p * n];
        u = csub(u, cmul(a, cconj(w)));
      }
      Uk[ii] = cdiv(u, piv);
    }
    __syncthreads();
    // v_k = conj(row); component scales and finiteness of u_k, v_k
    double cu = 0, cv = 0;
    bool bad = false;
    for (int ii = tid; ii < m; ii += nt) {
      const double2 u = Uk[ii];
      bad |= !isfinite(u.x) || !isfinite(u.y);
      cu = fmax(cu, fmax(fabs(u.x), fabs(u.y)));
    }
    for (int jj = tid; jj < n; jj += nt) {
      const double2 v = cconj(Vk[jj]);
      Vk[jj] = v;
      bad |= !isfinite(v.x) || !isfinite(v.y);
      cv = fmax(cv, fmax(fabs(v.x), fabs(v.y)));
    }
    double anybad = bad ? 1.0 : 0.0;
    block_max3(anybad, cu, cv, sh);
    if (anybad != 0.0) {
      status = 1;
      break;
    }
    if (!(cu > 0.0) || !(cv > 0.0)) {
      status = 2;
      break;
    }
    double su = 0, sv2 = 0;
    for (int ii = tid; ii < m; ii += nt) {
      const double xr = Uk[ii].x / cu, xi = Uk[ii].y / cu;
      su = fma(xr, xr, su);
      su = fma(xi, xi, su);
    }
    for (int jj = tid; jj < n; jj += nt) {
      const double xr = Vk[jj].x / cv, xi = Vk[jj].y / cv;
      sv2 = fma(xr, xr, sv2);
      sv2 = fma(xi, xi, sv2);
    }
    block_sum2(su, sv2, sh);
    // normalised inner products with the earlier factors: warp w takes the
    // ranks p = w, w + 8, ...
    for (int p = warp; p < k; p += nw) {
      const double2 *Up = U + (int64_t)p * m, *Vp = V + (int64_t)p * n;
      const double cup = S[p * ACA_SCR + 0], cvp = S[p * ACA_SCR + 2];
      double ur = 0, ui = 0, vr = 0, vi = 0;
      for (int ii = lane; ii < m; ii += 32) {
        const double lr = Up[ii].x / cup, li = Up[ii].y / cup, rr = Uk[ii].x / cu, ri2 = Uk[ii].y / cu;
        ur = fma(lr, rr, ur);
        ur = fma(li, ri2, ur);
        ui = fma(lr, ri2, ui);
        ui = fma(-li, rr, ui);
      }
      for (int jj = lane; jj < n; jj += 32) {
        const double lr = Vp[jj].x / cvp, li = Vp[jj].y / cvp, rr = Vk[jj].x / cv, ri2 = Vk[jj].y / cv;
        vr = fma(lr, rr, vr);
        vr = fma(li, ri2, vr);
        vi = fma(lr, ri2, vi);
        vi = fma(-li, rr, vi);
      }
      ur = warp_sum(ur);
      ui = warp_sum(ui);
      vr = warp_sum(vr);
      vi = warp_sum(vi);
      if (lane == 0) {
        S[p * ACA_SCR + 6] = ur;
        S[p * ACA_SCR + 7] = ui;
        S[p * ACA_SCR + 8] = vr;
        S[p * ACA_SCR + 9] = vi;
      }
    }
    __syncthreads();
    if (tid == 0) {
      const double nu = sqrt(su), nv = sqrt(sv2);
      Mag mu = mag_make(cu), mvv = mag_make(cv);
      Mag mun = mag_make(mu.f * nu), mvn = mag_make(mvv.f * nv);
      mun.e += mu.e;
      mvn.e += mvv.e;
      const Mag term = mag_mul(mun, mvn);
      double *Sk = S + k * ACA_SCR;
      Sk[0] = cu;
      Sk[1] = nu;
      Sk[2] = cv;
      Sk[3] = nv;
      Sk[4] = term.f;
      Sk[5] = (double)term.e;
      urow[prow] = 1;
      ucol[pc] = 1;
      if (k == 0) {
        fscale = term;
      } else if (mag_less(fscale, term)) {
        const double r = mag_ratio(fscale, term);
        fsq *= r * r;
        fscale = term;
      }
      const double tr = mag_ratio(term, fscale);
      double cross = 0.0;
      for (int p = 0; p < k; p++) {
        const double *Sp = S + p * ACA_SCR;
        const Mag tp{Sp[4], (int)Sp[5]};
        const double pr = mag_ratio(tp, fscale);
        const double un = Sp[1] * nu, vn = Sp[3] * nv;
        const double2 uc = make_double2(Sp[6] / un, Sp[7] / un), vc = make_double2(Sp[8] / vn, Sp[9] / vn);
        cross += 2.0 * pr * tr * (uc.x * vc.x + uc.y * vc.y);  // Re(uc conj(vc))
      }
      fsq += tr * tr + cross;
      fsq = fmax(fsq, 0.0);
      s_conv = tr < tol * sqrt(fsq) ? 1 : 0;
    }
    __syncthreads();
    rank = k + 1;
    if (s_conv) {
      converged = true;
      break;
    }
    // next pivot row: largest |u_k| among unused rows
    best = 0.0;
    bidx = -1;
    for (int ii = tid; ii < m; ii += nt) {
      const double au = hypot(Uk[ii].x, Uk[ii].y);
      if (!urow[ii] && au > best) {
        best = au;
        bidx = ii;
      }
    }
    block_argmax(best, bidx, sv, si);
    if (bidx < 0) break;
    prow = bidx;
  }
  if (tid == 0) {
    rank_out[bi] = rank;
    status_out[bi] = status;
    conv_out[bi] = converged ? 1 : 0;
  }
}

// ---------------------------------------------------------------------------
// device: H-matrix product
// ---------------------------------------------------------------------------
__global__ void k_aca_gather(int64_t N, const int *__restrict__ perm, const double2 *__restrict__ x,
                             double2 *__restrict__ xp) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) xp[i] = x[perm[i]];
}

// t_b = V_b^H x_cols (mode 0), U_b^H x_rows (1) or U_b^T x_rows (2)
__global__ void __launch_bounds__(256) k_aca_inner(const AcaBlockDesc *__restrict__ blocks, const int *__restrict__ lr,
                                                   const int *__restrict__ rank, const int64_t *__restrict__ toff,
                                                   const double2 *__restrict__ arena, const double2 *__restrict__ xp,
                                                   int mode, double2 *__restrict__ t) {
  const int b = lr[blockIdx.x];
  const AcaBlockDesc bd = blocks[b];
  const int r = rank[b];
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const bool fwd = mode == 0;
  const int len = fwd ? bd.n : bd.m;
  const double2 *F = arena + (fwd ? bd.off_b : bd.off_a);
  const double2 *xs = xp + (fwd ? bd.c0 : bd.r0);
  for (int p = threadIdx.x >> 5; p < r; p += nw) {
    const double2 *Fp = F + (int64_t)p * len;
    double2 acc = make_double2(0, 0);
#pragma unroll 4
    for (int i = lane; i < len; i += 32) {
      const double2 f = mode == 2 ? Fp[i] : cconj(Fp[i]);
      acc = cadd(acc, cmul(f, xs[i]));
    }
    acc = warp_sum2(acc);
    if (lane == 0) t[toff[b] + p] = acc;
  }
}

// Partial product of every block (one CTA each).  mode 0: z_b = D_b x_cols
// (dense) or U_b t_b (low-rank), m_b entries at zoff[b]; mode 1 / 2: the
// column side, n_b entries: D_b^H x_rows / D_b^T x_rows, or V_b t_b /
// conj(V_b) t_b.
__global__ void __launch_bounds__(256) k_aca_partials(const AcaBlockDesc *__restrict__ blocks,
                                                      const int *__restrict__ rank, const int64_t *__restrict__ toff,
                                                      const int64_t *__restrict__ zoff,
                                                      const double2 *__restrict__ arena,
                                                      const double2 *__restrict__ xp, const double2 *__restrict__ t,
                                                      int mode, double2 *__restrict__ z) {
  __shared__ double2 part[256];
  const int b = blockIdx.x;
  const AcaBlockDesc bd = blocks[b];
  double2 *zb = z + zoff[b];
  const int tid = threadIdx.x;
  if (mode == 0) {
    if (bd.kind == 0) {
      // 64 rows x 4 column groups per pass; the groups are summed in order
      const double2 *D = arena + bd.off_a, *xs = xp + bd.c0;
      const int ri = tid & 63, g = tid >> 6;
      for (int i0 = 0; i0 < bd.m; i0 += 64) {
        const int i = i0 + ri;
        double2 acc = make_double2(0, 0);
        if (i < bd.m) {
#pragma unroll 4
          for (int jj = g; jj < bd.n; jj += 4) acc = cadd(acc, cmul(D[i + (int64_t)jj * bd.m], xs[jj]));
        }
        part[tid] = acc;
        __syncthreads();
        if (tid < 64 && i < bd.m)
          zb[i] = cadd(cadd(part[tid], part[tid + 64]), cadd(part[tid + 128], part[tid + 192]));
        __syncthreads();
      }
    } else {
      const double2 *U = arena + bd.off_a, *tb = t + toff[b];
      const int r = rank[b];
      for (int i = tid; i < bd.m; i += blockDim.x) {
        double2 acc = make_double2(0, 0);
#pragma unroll 4
        for (int p = 0; p < r; p++) acc = cadd(acc, cmul(U[i + (int64_t)p * bd.m], tb[p]));
        zb[i] = acc;
      }
    }
    return;
  }
  const bool adj = mode == 1;
  if (bd.kind == 0) {
    // a warp per column: the column is contiguous in the block
    const double2 *D = arena + bd.off_a, *xs = xp + bd.r0;
    const int lane = tid & 31, nw = blockDim.x >> 5;
    for (int jj = tid >> 5; jj < bd.n; jj += nw) {
      const double2 *Dj = D + (int64_t)jj * bd.m;
      double2 acc = make_double2(0, 0);
#pragma unroll 2
      for (int ii = lane; ii < bd.m; ii += 32) acc = cadd(acc, cmul(adj ? cconj(Dj[ii]) : Dj[ii], xs[ii]));
      acc = warp_sum2(acc);
      if (lane == 0) zb[jj] = acc;
    }
  } else {
    const double2 *V = arena + bd.off_b, *tb = t + toff[b];
    const int r = rank[b];
    for (int j = tid; j < bd.n; j += blockDim.x) {
      double2 acc = make_double2(0, 0);
#pragma unroll 4
      for (int p = 0; p < r; p++) {
        const double2 v = V[j + (int64_t)p * bd.n];
        acc = cadd(acc, cmul(adj ? v : cconj(v), tb[p]));
      }
      zb[j] = acc;
    }
  }
}

// y over one leaf: the partial products of the blocks covering it, summed in
// the leaf's item order, scattered to the original order.  zbase[q] = the
// item's partial-product offset minus the block's first row (or column), so
// row i of the leaf reads z[zbase[q] + i].
__global__ void __launch_bounds__(64) k_aca_leaf_sum(const int2 *__restrict__ leaf, const int64_t *__restrict__ off,
                                                     const int64_t *__restrict__ zbase,
                                                     const double2 *__restrict__ z, const int *__restrict__ perm,
                                                     double2 *__restrict__ y) {
  const int2 L = leaf[blockIdx.x];
  const int64_t q0 = off[blockIdx.x], q1 = off[blockIdx.x + 1];
  for (int i = L.x + threadIdx.x; i < L.x + L.y; i += blockDim.x) {
    double2 acc = make_double2(0, 0);
    int64_t q = q0;
    for (; q + 4 <= q1; q += 4) {  // four independent loads in flight
      const double2 a = z[zbase[q] + i], b = z[zbase[q + 1] + i], c = z[zbase[q + 2] + i], d = z[zbase[q + 3] + i];
      acc = cadd(cadd(cadd(cadd(acc, a), b), c), d);
    }
    for (; q < q1; q++) acc = cadd(acc, z[zbase[q] + i]);
    y[perm[i]] = acc;
  }
}

// near-field matrix from the dense blocks (original index order)
template <class FC>
__global__ void k_aca_nf_scatter(const AcaBlockDesc *__restrict__ blocks, const int *__restrict__ ids,
                                 const int *__restrict__ perm, const double2 *__restrict__ arena, int64_t N,
                                 FC *__restrict__ F) {
  const AcaBlockDesc bd = blocks[ids[blockIdx.x]];
  const double2 *D = arena + bd.off_a;
  const int64_t cnt = (int64_t)bd.m * bd.n;
  for (int64_t e = threadIdx.x; e < cnt; e += blockDim.x) {
    const int ii = (int)(e % bd.m), jj = (int)(e / bd.m);
    store_c(F + (int64_t)perm[bd.r0 + ii] * N + perm[bd.c0 + jj], D[e]);
  }
}

__global__ void k_aca_diag_max(int64_t N, const double2 *__restrict__ d, double *__restrict__ out,
                               unsigned *__restrict__ bad) {
  __shared__ double red[32];
  double mx = 0;
  for (int64_t i = threadIdx.x; i < N; i += blockDim.x) {
    double a = hypot(d[i].x, d[i].y);
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

// _build_diagonal_preconditioner_data: 1 / Z_ii with |Z_ii| floored at
// 1e-10 max |Z_ii|
__global__ void k_aca_diag_inv(int64_t N, const double2 *__restrict__ d, const double *__restrict__ maxabs,
                               double2 *__restrict__ dinv) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double floor_abs = 1e-10 * (*maxabs);
  if (floor_abs == 0.0) floor_abs = 4.9406564584124654e-324;
  double2 z = d[i];
  if (hypot(z.x, z.y) < floor_abs) z = make_double2(floor_abs, 0);
  dinv[i] = cdiv(make_double2(1, 0), z);
}

AcaGeo make_geo(dmb_ctx *c) {
  AcaGeo g;
  g.tc = c->d_tcache.as<TriCache>();
  g.rslot = c->d_rwg_slot.as<int>();
  g.aoff = c->d_adj_off.as<int>();
  g.anb = c->d_adj_nb.as<int>();
  g.near_mn = c->d_near_entry_mn.as<int2>();
  g.near_off = c->d_near_entry_off.as<int64_t>();
  g.near_val = c->d_near_val.as<double2>();
  g.n_near = c->n_near_entry;
  g.k = c->aca.k;
  g.inv_k2 = 1.0 / (c->aca.k * c->aca.k);
  g.omega_mu0 = c->aca.k * c->aca.eta0;
  return g;
}

template <class T> void upload(dmb_ctx *c, DevBuf &b, const std::vector<T> &v) {
  b.ensure(std::max<size_t>(16, v.size() * sizeof(T)));
  if (!v.empty()) DMB_CUDA(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
}

#define ACA_NQ_DISPATCH(NQV, CALL)                  \
  switch (NQV) {                                    \
    case 1: { constexpr int NQ = 1; CALL; } break;  \
    case 3: { constexpr int NQ = 3; CALL; } break;  \
    case 4: { constexpr int NQ = 4; CALL; } break;  \
    default: { constexpr int NQ = 7; CALL; } break; \
  }

// dense fill of the listed blocks
void fill_dense(dmb_ctx *c, const std::vector<int> &ids) {
  if (ids.empty()) return;
  DevBuf d_ids;
  upload(c, d_ids, ids);
  AcaGeo g = make_geo(c);
  AcaState &A = c->aca;
  ACA_NQ_DISPATCH(c->nq, DMB_LAUNCH(c, k_aca_dense<NQ>, (unsigned)ids.size(), 256, 0, g,
                                    A.d_blocks.as<AcaBlockDesc>(), d_ids.as<int>(), A.d_perm.as<int>(),
                                    A.d_arena.as<double2>()));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
}

// leaf CSR lists: for each leaf the blocks whose row (by_row) or column range
// covers it, dense blocks first, each group in task order
void build_leaf_lists(const std::vector<AcaBlockDesc> &B, const std::vector<int2> &leaves, bool by_row,
                      std::vector<int64_t> &off, std::vector<int> &items) {
  const int64_t nl = (int64_t)leaves.size();
  std::vector<int> starts(nl);
  for (int64_t l = 0; l < nl; l++) starts[l] = leaves[l].x;
  std::vector<std::vector<int>> lists(nl);
  for (int pass = 0; pass < 2; pass++)
    for (size_t b = 0; b < B.size(); b++) {
      if ((pass == 0) != (B[b].kind == 0)) continue;
      const int lo = by_row ? B[b].r0 : B[b].c0, cnt = by_row ? B[b].m : B[b].n;
      int64_t l = std::upper_bound(starts.begin(), starts.end(), lo) - starts.begin() - 1;
      for (; l < nl && leaves[l].x < lo + cnt; l++) lists[l].push_back((int)b);
    }
  off.assign(nl + 1, 0);
  for (int64_t l = 0; l < nl; l++) off[l + 1] = off[l] + (int64_t)lists[l].size();
  items.clear();
  items.reserve(off[nl]);
  for (auto &v : lists) items.insert(items.end(), v.begin(), v.end());
}

// ACA launch of one size bucket (count blocks from ids / foff / soff)
template <int NT>
void launch_lowrank(dmb_ctx *c, unsigned count, const AcaGeo &g, const AcaBlockDesc *blocks, const int *ids,
                    const int *perm, double2 *arena, const int64_t *foff, unsigned char *flags, const int64_t *soff,
                    double *scr, double tol, int *rank, int *status, int *conv) {
  if (count == 0) return;
  ACA_NQ_DISPATCH(c->nq, DMB_LAUNCH(c, (k_aca_lowrank<NQ, NT>), count, NT, 0, g, blocks, ids, perm, arena, foff,
                                    flags, soff, scr, tol, rank, status, conv));
}

void ensure_side_streams(dmb_ctx *c) {
  if (!c->stream2 || !c->stream3) {
    int least = 0, greatest = 0;
    DMB_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    // the same priorities as the factorisation's lookahead streams
    const int mid = greatest < least ? greatest + 1 : least;
    if (!c->stream2) DMB_CUDA(cudaStreamCreateWithPriority(&c->stream2, cudaStreamNonBlocking, mid));
    if (!c->stream3) DMB_CUDA(cudaStreamCreateWithPriority(&c->stream3, cudaStreamNonBlocking, mid));
  }
  for (auto &e : c->la_ev)
    if (!e) DMB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
}

}  // namespace

namespace dmb {

bool operator_ready(dmb_ctx *c) { return c->op_kind == 1 ? c->aca.valid : c->z_valid; }

void aca_build(dmb_ctx *c, double k, double eta0, int quad_order, int leaf_size, double eta, double tol,
               int max_rank, int64_t max_tasks, int64_t max_storage, dmb_aca_info *info) {
  const double t0 = now_ms();
  DMB_REQUIRE(std::isfinite(k) && k != 0.0, DMB_ERR_ARGUMENT, "EFIE wavenumber must be finite and nonzero");
  DMB_REQUIRE(std::isfinite(eta0) && eta0 != 0.0, DMB_ERR_ARGUMENT, "EFIE eta0 must be finite and nonzero");
  DMB_REQUIRE(std::isfinite(tol) && tol > 0.0, DMB_ERR_ARGUMENT,
              "ACA tolerance must be finite and positive, got " + std::to_string(tol));
  DMB_REQUIRE(max_rank >= 1, DMB_ERR_ARGUMENT, "ACA max_rank must be at least 1, got " + std::to_string(max_rank));
  DMB_REQUIRE(max_storage >= 1, DMB_ERR_ARGUMENT,
              "max_storage_bytes must be positive, got " + std::to_string(max_storage));
  const double inv_k2 = 1.0 / (k * k);
  DMB_REQUIRE(std::isfinite(inv_k2) && std::isfinite(k * eta0) && k * eta0 != 0.0, DMB_ERR_OVERFLOW,
              "EFIE prefactors are not representable");
  AcaState &A = c->aca;
  A.release();
  c->op_kind = 0;
  prepare_operator(c, k, eta0, quad_order);  // triangle cache + near records for this k
  const int64_t N = c->n;
  // plan on the RWG centres of the device cache
  std::vector<double> ctr(3 * N);
  DMB_CUDA(cudaMemcpyAsync(ctr.data(), c->d_centers.p, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, c->stream));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  Plan P;
  make_plan(ctr.data(), N, leaf_size, eta, max_tasks, P);
  const double t_plan = now_ms();
  // _validate_aca_task_storage (src/fast/ACA.jl:740-772)
  double planned = 0;
  for (const Task &t : P.tasks) {
    const double m = (double)(P.nodes[t.row].hi - P.nodes[t.row].lo + 1);
    const double n = (double)(P.nodes[t.col].hi - P.nodes[t.col].lo + 1);
    planned += t.kind == 0 ? m * n : std::min<double>(max_rank, std::min(m, n)) * (m + n);
  }
  const double planned_bytes = planned * 16.0;
  DMB_REQUIRE(planned_bytes <= (double)max_storage, DMB_ERR_ARGUMENT,
              "ACA block storage requires at most " + std::to_string((int64_t)planned_bytes) +
                  " raw bytes, exceeding max_storage_bytes=" + std::to_string(max_storage));
  // block descriptors in task order and the arena
  A.n = N;
  A.k = k;
  A.eta0 = eta0;
  A.quad_order = quad_order;
  A.perm.resize(N);
  for (int64_t i = 0; i < N; i++) A.perm[i] = (int32_t)P.perm[i];
  A.blocks.resize(P.tasks.size());
  int64_t off = 0;
  std::vector<int> dense_ids, lr_ids;
  for (size_t b = 0; b < P.tasks.size(); b++) {
    const Task &t = P.tasks[b];
    AcaBlockDesc &d = A.blocks[b];
    d.r0 = (int32_t)P.nodes[t.row].lo;
    d.m = (int32_t)(P.nodes[t.row].hi - P.nodes[t.row].lo + 1);
    d.c0 = (int32_t)P.nodes[t.col].lo;
    d.n = (int32_t)(P.nodes[t.col].hi - P.nodes[t.col].lo + 1);
    d.kind = t.kind;
    d.task = (int32_t)b;
    d.fallback = 0;
    if (t.kind == 0) {
      d.rmax = 0;
      d.off_a = off;
      d.off_b = 0;
      off += (int64_t)d.m * d.n;
      dense_ids.push_back((int)b);
    } else {
      d.rmax = std::min(max_rank, std::min(d.m, d.n));
      d.off_a = off;
      d.off_b = off + (int64_t)d.m * d.rmax;
      off += (int64_t)d.rmax * (d.m + d.n);
      lr_ids.push_back((int)b);
    }
  }
  A.d_arena.ensure(sizeof(double2) * std::max<int64_t>(off, 1));
  std::vector<int32_t> perm32(A.perm.begin(), A.perm.end());
  upload(c, A.d_perm, perm32);
  upload(c, A.d_blocks, A.blocks);
  fill_dense(c, dense_ids);
  const double t_dense = now_ms();
  // ACA on every admissible block, largest first (the CTAs of the big blocks
  // start in the first wave)
  std::vector<int> rank(A.blocks.size(), 0), status(A.blocks.size(), 0), conv(A.blocks.size(), 1);
  if (!lr_ids.empty()) {
    // largest first; buckets by m + n: 512-thread CTAs for the few large
    // blocks (the critical path), 256 for the middle, 64 for the many
    // leaf-level blocks, launched concurrently on the context's three streams
    std::vector<int> order = lr_ids;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
      const AcaBlockDesc &x = A.blocks[a], &y = A.blocks[b];
      return x.m + x.n != y.m + y.n ? x.m + x.n > y.m + y.n : x.rmax > y.rmax;
    });
    size_t e512 = 0, e256 = 0;
    while (e512 < order.size() && A.blocks[order[e512]].m + A.blocks[order[e512]].n > 1024) e512++;
    e256 = e512;
    while (e256 < order.size() && A.blocks[order[e256]].m + A.blocks[order[e256]].n > 192) e256++;
    std::vector<int64_t> foff(order.size()), soff(order.size());
    int64_t fo = 0, so = 0;
    for (size_t q = 0; q < order.size(); q++) {
      const AcaBlockDesc &d = A.blocks[order[q]];
      foff[q] = fo;
      soff[q] = so;
      fo += d.m + d.n;
      so += (int64_t)ACA_SCR * d.rmax;
    }
    DevBuf d_ids, d_foff, d_soff, d_flags, d_scr, d_rank, d_status, d_conv;
    upload(c, d_ids, order);
    upload(c, d_foff, foff);
    upload(c, d_soff, soff);
    d_flags.ensure(std::max<int64_t>(fo, 16));
    DMB_CUDA(cudaMemsetAsync(d_flags.p, 0, std::max<int64_t>(fo, 16), c->stream));
    d_scr.ensure(sizeof(double) * std::max<int64_t>(so, 2));
    d_rank.ensure(sizeof(int) * A.blocks.size());
    d_status.ensure(sizeof(int) * A.blocks.size());
    d_conv.ensure(sizeof(int) * A.blocks.size());
    DMB_CUDA(cudaMemsetAsync(d_rank.p, 0, sizeof(int) * A.blocks.size(), c->stream));
    DMB_CUDA(cudaMemsetAsync(d_status.p, 0, sizeof(int) * A.blocks.size(), c->stream));
    DMB_CUDA(cudaMemsetAsync(d_conv.p, 0, sizeof(int) * A.blocks.size(), c->stream));
    AcaGeo g = make_geo(c);
    ensure_side_streams(c);
    DMB_CUDA(cudaEventRecord(c->la_ev[0], c->stream));
    DMB_CUDA(cudaStreamWaitEvent(c->stream2, c->la_ev[0], 0));
    DMB_CUDA(cudaStreamWaitEvent(c->stream3, c->la_ev[0], 0));
    auto bucket = [&](auto nt_tag, size_t lo, size_t hi) {
      constexpr int NT = decltype(nt_tag)::value;
      launch_lowrank<NT>(c, (unsigned)(hi - lo), g, A.d_blocks.as<AcaBlockDesc>(), d_ids.as<int>() + lo,
                         A.d_perm.as<int>(), A.d_arena.as<double2>(), d_foff.as<int64_t>() + lo,
                         d_flags.as<unsigned char>(), d_soff.as<int64_t>() + lo, d_scr.as<double>(), tol,
                         d_rank.as<int>(), d_status.as<int>(), d_conv.as<int>());
    };
    bucket(std::integral_constant<int, 512>(), 0, e512);
    {
      StreamSwap sw(c, c->stream2);
      bucket(std::integral_constant<int, 256>(), e512, e256);
      DMB_CUDA(cudaEventRecord(c->la_ev[1], c->stream2));
    }
    {
      StreamSwap sw(c, c->stream3);
      bucket(std::integral_constant<int, 64>(), e256, order.size());
      DMB_CUDA(cudaEventRecord(c->la_ev[2], c->stream3));
    }
    DMB_CUDA(cudaStreamWaitEvent(c->stream, c->la_ev[1], 0));
    DMB_CUDA(cudaStreamWaitEvent(c->stream, c->la_ev[2], 0));
    DMB_CUDA(cudaMemcpyAsync(rank.data(), d_rank.p, sizeof(int) * rank.size(), cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaMemcpyAsync(status.data(), d_status.p, sizeof(int) * status.size(), cudaMemcpyDeviceToHost,
                             c->stream));
    DMB_CUDA(cudaMemcpyAsync(conv.data(), d_conv.p, sizeof(int) * conv.size(), cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
  }
  const double t_lowrank = now_ms();
  // non-finite updates: the block is stored dense (src/fast/ACA.jl:883-946),
  // within the storage budget
  std::vector<int> fb;
  for (int b : lr_ids) {
    DMB_REQUIRE(status[b] != 2, DMB_ERR_OVERFLOW, "ACA low-rank update has zero norm");
    if (status[b] == 1) fb.push_back(b);
  }
  if (!fb.empty()) {
    double claimed = planned_bytes;
    int64_t extra = 0;
    for (int b : fb) {
      const AcaBlockDesc &d = A.blocks[b];
      const double dense = (double)d.m * d.n, plan = (double)d.rmax * (d.m + d.n);
      const double xb = std::max(0.0, dense - plan) * 16.0;
      DMB_REQUIRE(xb <= (double)max_storage - claimed, DMB_ERR_ARGUMENT,
                  "ACA dense fallback would exceed max_storage_bytes=" + std::to_string(max_storage));
      claimed += xb;
      extra += (int64_t)d.m * d.n;
    }
    // grow the arena: copy the existing data into a larger one
    DevBuf bigger;
    bigger.ensure(sizeof(double2) * (off + extra));
    DMB_CUDA(cudaMemcpyAsync(bigger.p, A.d_arena.p, sizeof(double2) * off, cudaMemcpyDeviceToDevice, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
    std::swap(bigger.p, A.d_arena.p);
    std::swap(bigger.bytes, A.d_arena.bytes);
    bigger.release();
    for (int b : fb) {
      AcaBlockDesc &d = A.blocks[b];
      d.kind = 0;
      d.fallback = 1;
      d.off_a = off;
      d.off_b = 0;
      off += (int64_t)d.m * d.n;
      rank[b] = 0;
    }
    upload(c, A.d_blocks, A.blocks);
    fill_dense(c, fb);
  }
  A.rank.assign(rank.begin(), rank.end());
  // product lists
  std::vector<int2> leaves;
  for (const Node &nd : P.nodes)
    if (nd.left < 0) leaves.push_back(make_int2((int)nd.lo, (int)(nd.hi - nd.lo + 1)));
  std::sort(leaves.begin(), leaves.end(), [](int2 a, int2 b) { return a.x < b.x; });
  A.n_leaves = (int64_t)leaves.size();
  std::vector<int> lr_now;
  std::vector<int64_t> toff(A.blocks.size(), 0);
  int64_t tt = 0;
  int64_t stored = 0, n_dense = 0, max_r = 0, uncv = 0;
  for (size_t b = 0; b < A.blocks.size(); b++) {
    const AcaBlockDesc &d = A.blocks[b];
    if (d.kind == 1) {
      lr_now.push_back((int)b);
      toff[b] = tt;
      tt += std::max(1, rank[b]);
      stored += (int64_t)rank[b] * (d.m + d.n);
      max_r = std::max<int64_t>(max_r, rank[b]);
      if (!conv[b] && rank[b] == d.rmax && d.rmax < std::min(d.m, d.n)) uncv++;
    } else {
      n_dense++;
      stored += (int64_t)d.m * d.n;
    }
  }
  A.n_lr = (int64_t)lr_now.size();
  A.t_total = tt;
  std::vector<int64_t> roff, coff;
  std::vector<int> ritems, citems;
  build_leaf_lists(A.blocks, leaves, true, roff, ritems);
  build_leaf_lists(A.blocks, leaves, false, coff, citems);
  upload(c, A.d_leaf, leaves);
  upload(c, A.d_row_off, roff);
  upload(c, A.d_col_off, coff);
  upload(c, A.d_lr_list, lr_now);
  upload(c, A.d_tbuf_off, toff);
  // partial-product offsets: row side and column side of every block
  std::vector<int64_t> zr(A.blocks.size()), zc(A.blocks.size());
  int64_t sr = 0, sc = 0;
  for (size_t b = 0; b < A.blocks.size(); b++) {
    zr[b] = sr;
    zc[b] = sc;
    sr += A.blocks[b].m;
    sc += A.blocks[b].n;
  }
  upload(c, A.d_zoff_r, zr);
  upload(c, A.d_zoff_c, zc);
  std::vector<int64_t> rzb(ritems.size()), czb(citems.size());
  for (size_t q = 0; q < ritems.size(); q++) rzb[q] = zr[ritems[q]] - A.blocks[ritems[q]].r0;
  for (size_t q = 0; q < citems.size(); q++) czb[q] = zc[citems[q]] - A.blocks[citems[q]].c0;
  upload(c, A.d_row_zbase, rzb);
  upload(c, A.d_col_zbase, czb);
  A.d_z.ensure(sizeof(double2) * std::max<int64_t>(1, std::max(sr, sc)));
  std::vector<int32_t> rk(rank.begin(), rank.end());
  upload(c, A.d_rank, rk);
  A.d_t.ensure(sizeof(double2) * std::max<int64_t>(tt, 1));
  A.d_xp.ensure(sizeof(double2) * N);
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  A.info = dmb_aca_info{};
  A.info.n_dense = n_dense;
  A.info.n_lowrank = A.n_lr;
  A.info.n_fallback = (int64_t)fb.size();
  A.info.max_rank_used = max_r;
  A.info.entries_stored = stored;
  A.info.n_unconverged = uncv;
  A.info.build_ms = now_ms() - t0;
  A.info.plan_ms = t_plan - t0;
  A.info.dense_ms = t_dense - t_plan;
  A.info.lowrank_ms = t_lowrank - t_dense;
  A.valid = true;
  c->op_kind = 1;
  c->aca_transposed = false;
  c->pc_valid = false;
  if (info) *info = A.info;
}

void aca_apply(dmb_ctx *c, const double2 *x, double2 *y, int64_t nrhs, int mode) {
  AcaState &A = c->aca;
  DMB_REQUIRE(A.valid, DMB_ERR_STATE, "no H-matrix operator built");
  DMB_REQUIRE(mode >= 0 && mode <= 2, DMB_ERR_ARGUMENT, "ACA product mode must be 0, 1 or 2");
  const int64_t N = A.n;
  // algorithmic bytes of one product: every stored block entry once, x and y
  const double bytes = 16.0 * ((double)A.info.entries_stored + 2.0 * (double)N);
  for (int64_t r = 0; r < nrhs; r++) {
    const double2 *xr = x + r * N;
    double2 *yr = y + r * N;
    kt_begin(c);
    DMB_LAUNCH(c, k_aca_gather, blocks_for(N, 256), 256, 0, N, A.d_perm.as<int>(), xr, A.d_xp.as<double2>());
    if (A.n_lr > 0)
      DMB_LAUNCH(c, k_aca_inner, (unsigned)A.n_lr, 256, 0, A.d_blocks.as<AcaBlockDesc>(), A.d_lr_list.as<int>(),
                 A.d_rank.as<int>(), A.d_tbuf_off.as<int64_t>(), A.d_arena.as<double2>(), A.d_xp.as<double2>(), mode,
                 A.d_t.as<double2>());
    DMB_LAUNCH(c, k_aca_partials, (unsigned)A.blocks.size(), 256, 0, A.d_blocks.as<AcaBlockDesc>(),
               A.d_rank.as<int>(), A.d_tbuf_off.as<int64_t>(),
               (mode == 0 ? A.d_zoff_r : A.d_zoff_c).as<int64_t>(), A.d_arena.as<double2>(), A.d_xp.as<double2>(),
               A.d_t.as<double2>(), mode, A.d_z.as<double2>());
    if (mode == 0)
      DMB_LAUNCH(c, k_aca_leaf_sum, (unsigned)A.n_leaves, 64, 0, A.d_leaf.as<int2>(), A.d_row_off.as<int64_t>(),
                 A.d_row_zbase.as<int64_t>(), A.d_z.as<double2>(), A.d_perm.as<int>(), yr);
    else
      DMB_LAUNCH(c, k_aca_leaf_sum, (unsigned)A.n_leaves, 64, 0, A.d_leaf.as<int2>(), A.d_col_off.as<int64_t>(),
                 A.d_col_zbase.as<int64_t>(), A.d_z.as<double2>(), A.d_perm.as<int>(), yr);
    kt_end(c, bytes, 3);
  }
}

void nf_factor_resident(dmb_ctx *c, int kind, int precision);
void refresh_geo(dmb_ctx *c);

void aca_nf_build(dmb_ctx *c, int kind, int precision) {
  AcaState &A = c->aca;
  DMB_REQUIRE(A.valid, DMB_ERR_STATE, "no H-matrix operator built");
  DMB_REQUIRE(kind == DMB_PRECOND_NF_LU || kind == DMB_PRECOND_NF_DIAG, DMB_ERR_ARGUMENT,
              "invalid factorization; expected :lu or :diag");
  DMB_REQUIRE(precision == DMB_PREC_FP64 || precision == DMB_PREC_MIXED, DMB_ERR_ARGUMENT,
              "precision must be DMB_PREC_FP64 or DMB_PREC_MIXED");
  const double t0 = now_ms();
  const int64_t N = A.n;
  c->pc_valid = false;
  std::vector<int> dense;
  int64_t nnz = 0;
  for (size_t b = 0; b < A.blocks.size(); b++)
    if (A.blocks[b].kind == 0) {
      dense.push_back((int)b);
      nnz += (int64_t)A.blocks[b].m * A.blocks[b].n;
    }
  if (kind == DMB_PRECOND_NF_DIAG) {
    refresh_geo(c);
    // the diagonal entries lie in the dense blocks (a cluster is never
    // admissible against itself); evaluate them directly
    std::vector<int> mn(2 * N);
    for (int64_t i = 0; i < N; i++) mn[2 * i] = mn[2 * i + 1] = (int)i;
    DevBuf d_mn, d_diag, tmp;
    upload(c, d_mn, mn);
    d_diag.ensure(sizeof(double2) * N);
    tmp.ensure(16);
    DMB_CUDA(cudaMemsetAsync(tmp.p, 0, 16, c->stream));
    AcaGeo g = make_geo(c);
    DMB_LAUNCH(c, k_aca_entries, blocks_for(N, 128), 128, 0, g, c->nq, N, d_mn.as<int>(), d_diag.as<double2>());
    c->d_dinv.ensure(sizeof(double2) * N);
    unsigned *bad = (unsigned *)(tmp.as<double>() + 1);
    DMB_LAUNCH(c, k_aca_diag_max, 1, 1024, 0, N, d_diag.as<double2>(), tmp.as<double>(), bad);
    DMB_LAUNCH(c, k_aca_diag_inv, blocks_for(N, 256), 256, 0, N, d_diag.as<double2>(), tmp.as<double>(),
               c->d_dinv.as<double2>());
    double mx[2];
    DMB_CUDA(cudaMemcpyAsync(mx, tmp.p, 16, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
    unsigned hb;
    memcpy(&hb, &mx[1], 4);
    DMB_REQUIRE(hb == 0, DMB_ERR_ARGUMENT, "near-field diagonal entries must be finite");
    DMB_REQUIRE(mx[0] > 0, DMB_ERR_ARGUMENT, "cannot build a diagonal preconditioner from an all-zero diagonal");
    c->nnz_ratio = 1.0 / (double)N;
    c->pc_kind = kind;
    c->pc_prec = precision;
    c->pc_valid = true;
    c->tm.precond_ms = now_ms() - t0;
    return;
  }
  const bool f64 = precision == DMB_PREC_FP64;
  const size_t esz = f64 ? sizeof(double2) : sizeof(float2);
  c->d_F.ensure(esz * N * N);
  DMB_CUDA(cudaMemsetAsync(c->d_F.p, 0, esz * N * N, c->stream));
  DevBuf d_ids;
  upload(c, d_ids, dense);
  if (!dense.empty()) {
    if (f64)
      DMB_LAUNCH(c, k_aca_nf_scatter<double2>, (unsigned)dense.size(), 256, 0, A.d_blocks.as<AcaBlockDesc>(),
                 d_ids.as<int>(), A.d_perm.as<int>(), A.d_arena.as<double2>(), N, c->d_F.as<double2>());
    else
      DMB_LAUNCH(c, k_aca_nf_scatter<float2>, (unsigned)dense.size(), 256, 0, A.d_blocks.as<AcaBlockDesc>(),
                 d_ids.as<int>(), A.d_perm.as<int>(), A.d_arena.as<double2>(), N, c->d_F.as<float2>());
  }
  c->nnz_ratio = ((double)nnz / (double)N) / (double)N;
  nf_factor_resident(c, kind, precision);
  c->tm.precond_ms = now_ms() - t0;
}

// the singular records of the operator's wavenumber (another build or a
// matrix-free set-up on this context may have replaced them)
void refresh_geo(dmb_ctx *c) {
  const AcaState &A = c->aca;
  if (c->k != A.k || c->eta0 != A.eta0 || !c->cache_valid || c->cache_quad_order != A.quad_order)
    prepare_operator(c, A.k, A.eta0, A.quad_order);
}

void aca_entries(dmb_ctx *c, const int64_t *m, const int64_t *n, int64_t count, double *out) {
  AcaState &A = c->aca;
  DMB_REQUIRE(A.valid, DMB_ERR_STATE, "no H-matrix operator built");
  refresh_geo(c);
  std::vector<int> mn(2 * count);
  for (int64_t e = 0; e < count; e++) {
    DMB_REQUIRE(m[e] >= 1 && m[e] <= A.n && n[e] >= 1 && n[e] <= A.n, DMB_ERR_ARGUMENT, "entry index out of range");
    mn[2 * e] = (int)(m[e] - 1);
    mn[2 * e + 1] = (int)(n[e] - 1);
  }
  DevBuf d_mn, d_out;
  upload(c, d_mn, mn);
  d_out.ensure(sizeof(double2) * std::max<int64_t>(count, 1));
  AcaGeo g = make_geo(c);
  if (count > 0)
    DMB_LAUNCH(c, k_aca_entries, blocks_for(count, 128), 128, 0, g, c->nq, count, d_mn.as<int>(),
               d_out.as<double2>());
  DMB_CUDA(cudaMemcpyAsync(out, d_out.p, sizeof(double2) * count, cudaMemcpyDeviceToHost, c->stream));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
}

// aca_lowrank(cache, rows, cols; tol, max_rank) (src/fast/ACA.jl:351-554) on
// one block of arbitrary RWG index lists (0-based); U m x r, V n x r to host
int aca_lowrank_one(dmb_ctx *c, double k, double eta0, int quad_order, const std::vector<int> &rows,
                    const std::vector<int> &cols, double tol, int max_rank, double *U_out, double *V_out) {
  const int m = (int)rows.size(), n = (int)cols.size();
  const int rmax = std::min(max_rank, std::min(m, n));
  prepare_operator(c, k, eta0, quad_order);
  // the kernel reads rows from perm[r0..] and columns from perm[c0..]
  std::vector<int> idx(rows);
  idx.insert(idx.end(), cols.begin(), cols.end());
  AcaBlockDesc d{};
  d.r0 = 0;
  d.m = m;
  d.c0 = m;
  d.n = n;
  d.kind = 1;
  d.rmax = rmax;
  d.off_a = 0;
  d.off_b = (int64_t)m * rmax;
  std::vector<AcaBlockDesc> blk = {d};
  std::vector<int> ids = {0};
  std::vector<int64_t> foff = {0}, soff = {0};
  DevBuf d_idx, d_blk, d_ids, d_foff, d_soff, d_arena, d_flags, d_scr, d_out;
  upload(c, d_idx, idx);
  upload(c, d_blk, blk);
  upload(c, d_ids, ids);
  upload(c, d_foff, foff);
  upload(c, d_soff, soff);
  d_arena.ensure(sizeof(double2) * std::max<int64_t>(1, (int64_t)rmax * (m + n)));
  d_flags.ensure(std::max(16, m + n));
  DMB_CUDA(cudaMemsetAsync(d_flags.p, 0, std::max(16, m + n), c->stream));
  d_scr.ensure(sizeof(double) * std::max(2, ACA_SCR * rmax));
  d_out.ensure(sizeof(int) * 3);
  DMB_CUDA(cudaMemsetAsync(d_out.p, 0, sizeof(int) * 3, c->stream));
  AcaGeo g = make_geo(c);
  g.k = k;
  g.inv_k2 = 1.0 / (k * k);
  g.omega_mu0 = k * eta0;
  int *o = d_out.as<int>();
  launch_lowrank<256>(c, 1, g, d_blk.as<AcaBlockDesc>(), d_ids.as<int>(), d_idx.as<int>(), d_arena.as<double2>(),
                      d_foff.as<int64_t>(), d_flags.as<unsigned char>(), d_soff.as<int64_t>(), d_scr.as<double>(),
                      tol, o, o + 1, o + 2);
  int h[3];
  DMB_CUDA(cudaMemcpyAsync(h, d_out.p, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  DMB_CUDA(cudaStreamSynchronize(c->stream));
  DMB_REQUIRE(h[1] != 1, DMB_ERR_OVERFLOW, "ACA low-rank update became non-finite");
  DMB_REQUIRE(h[1] != 2, DMB_ERR_OVERFLOW, "ACA low-rank update has zero norm");
  const int r = h[0];
  if (r > 0) {
    DMB_CUDA(cudaMemcpyAsync(U_out, d_arena.p, sizeof(double2) * m * r, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaMemcpyAsync(V_out, d_arena.as<double2>() + d.off_b, sizeof(double2) * n * r,
                             cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
  }
  return r;
}

}  // namespace dmb

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
namespace {
template <class F> dmb_status aca_guarded(dmb_ctx *c, F &&f) {
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
template <class F> dmb_status free_guarded(F &&f) {
  try {
    f();
    return DMB_OK;
  } catch (const DmbError &e) {
    dmb_free_error() = e.msg;
    return e.code;
  } catch (const std::exception &e) {
    dmb_free_error() = e.what();
    return DMB_ERR_STATE;
  }
}
}  // namespace

extern "C" {

dmb_status dmb_aca_plan(const double *centers, int64_t n, int leaf_size, double eta, int64_t max_block_tasks,
                        int64_t *perm_out, int64_t *n_nodes_out, int64_t *nodes_out, double *boxes_out,
                        int64_t *n_tasks_out, int64_t *tasks_out, int64_t tasks_cap) {
  return free_guarded([&] {
    DMB_REQUIRE(centers || n == 0, DMB_ERR_ARGUMENT, "centers is NULL");
    Plan P;
    make_plan(centers, n, leaf_size, eta, max_block_tasks, P);
    if (perm_out)
      for (int64_t i = 0; i < n; i++) perm_out[i] = P.perm[i] + 1;
    if (n_nodes_out) *n_nodes_out = (int64_t)P.nodes.size();
    for (size_t i = 0; i < P.nodes.size(); i++) {
      const Node &nd = P.nodes[i];
      if (nodes_out) {
        int64_t *o = nodes_out + 5 * i;
        o[0] = nd.lo + 1;
        o[1] = nd.hi + 1;
        o[2] = nd.left + 1;
        o[3] = nd.right + 1;
        o[4] = nd.level;
      }
      if (boxes_out)
        for (int c = 0; c < 3; c++) {
          boxes_out[6 * i + c] = nd.bmin[c];
          boxes_out[6 * i + 3 + c] = nd.bmax[c];
        }
    }
    if (n_tasks_out) *n_tasks_out = (int64_t)P.tasks.size();
    if (tasks_out && tasks_cap >= (int64_t)P.tasks.size())
      for (size_t t = 0; t < P.tasks.size(); t++) {
        int64_t *o = tasks_out + 5 * t;
        o[0] = P.tasks[t].row + 1;
        o[1] = P.tasks[t].col + 1;
        o[2] = P.tasks[t].kind;
        o[3] = 0;
        o[4] = 0;
      }
  });
}

dmb_status dmb_aca_admissible(const double *box_i, const double *box_j, double eta, int *out) {
  return free_guarded([&] {
    DMB_REQUIRE(box_i && box_j && out, DMB_ERR_ARGUMENT, "NULL argument");
    *out = box_admissible(box_i, box_i + 3, box_j, box_j + 3, eta) ? 1 : 0;
  });
}

dmb_status dmb_aca_build(dmb_ctx *c, double k, double eta0, int quad_order, int leaf_size, double eta,
                         double aca_tol, int max_rank, int64_t max_block_tasks, int64_t max_storage_bytes,
                         dmb_aca_info *info_out) {
  return aca_guarded(c, [&] {
    DMB_REQUIRE(c->have_mesh && c->have_rwg, DMB_ERR_STATE, "mesh and RWG data must be uploaded first");
    dmb::aca_build(c, k, eta0, quad_order, leaf_size, eta, aca_tol, max_rank, max_block_tasks, max_storage_bytes,
                   info_out);
  });
}

dmb_status dmb_aca_matvec(dmb_ctx *c, const double *x, double *y, int64_t nrhs, int mode) {
  return aca_guarded(c, [&] {
    DMB_REQUIRE(c->aca.valid, DMB_ERR_STATE, "no H-matrix operator built");
    DMB_REQUIRE(x && y && nrhs >= 1, DMB_ERR_ARGUMENT, "bad product arrays");
    for (int64_t i = 0; i < 2 * c->aca.n * nrhs; i++)
      DMB_REQUIRE(std::isfinite(x[i]), DMB_ERR_ARGUMENT, "x must contain only finite values");
    const size_t bytes = sizeof(double2) * c->aca.n * nrhs;
    DevBuf bx, by;
    bx.ensure(bytes);
    by.ensure(bytes);
    DMB_CUDA(cudaMemcpyAsync(bx.p, x, bytes, cudaMemcpyHostToDevice, c->stream));
    dmb::aca_apply(c, bx.as<double2>(), by.as<double2>(), nrhs, mode);
    DMB_CUDA(cudaMemcpyAsync(y, by.p, bytes, cudaMemcpyDeviceToHost, c->stream));
    DMB_CUDA(cudaStreamSynchronize(c->stream));
  });
}

dmb_status dmb_aca_blocks(dmb_ctx *c, int64_t *out) {
  return aca_guarded(c, [&] {
    DMB_REQUIRE(c->aca.valid, DMB_ERR_STATE, "no H-matrix operator built");
    DMB_REQUIRE(out, DMB_ERR_ARGUMENT, "output is NULL");
    const AcaState &A = c->aca;
    for (size_t b = 0; b < A.blocks.size(); b++) {
      const AcaBlockDesc &d = A.blocks[b];
      int64_t *o = out + 7 * b;
      o[0] = d.kind;
      o[1] = d.r0 + 1;
      o[2] = d.r0 + d.m;
      o[3] = d.c0 + 1;
      o[4] = d.c0 + d.n;
      o[5] = d.kind == 1 ? A.rank[b] : 0;
      o[6] = d.fallback;
    }
  });
}

dmb_status dmb_aca_block_data(dmb_ctx *c, int64_t b, double *a_out, double *b_out) {
  return aca_guarded(c, [&] {
    const AcaState &A = c->aca;
    DMB_REQUIRE(A.valid, DMB_ERR_STATE, "no H-matrix operator built");
    DMB_REQUIRE(b >= 0 && b < (int64_t)A.blocks.size(), DMB_ERR_ARGUMENT, "block index out of range");
    const AcaBlockDesc &d = A.blocks[b];
    const double2 *base = A.d_arena.as<double2>();
    if (d.kind == 0) {
      DMB_REQUIRE(a_out, DMB_ERR_ARGUMENT, "output is NULL");
      DMB_CUDA(cudaMemcpyAsync(a_out, base + d.off_a, sizeof(double2) * d.m * d.n, cudaMemcpyDeviceToHost,
                               c->stream));
    } else {
      DMB_REQUIRE(a_out && b_out, DMB_ERR_ARGUMENT, "output is NULL");
      const int64_t r = A.rank[b];
      if (r > 0) {
        DMB_CUDA(cudaMemcpyAsync(a_out, base + d.off_a, sizeof(double2) * d.m * r, cudaMemcpyDeviceToHost,
                                 c->stream));
        DMB_CUDA(cudaMemcpyAsync(b_out, base + d.off_b, sizeof(double2) * d.n * r, cudaMemcpyDeviceToHost,
                                 c->stream));
      }
    }
    DMB_CUDA(cudaStreamSynchronize(c->stream));
  });
}

dmb_status dmb_aca_entries(dmb_ctx *c, const int64_t *m, const int64_t *n, int64_t count, double *out) {
  return aca_guarded(c, [&] {
    DMB_REQUIRE((m && n && out) || count == 0, DMB_ERR_ARGUMENT, "NULL argument");
    dmb::aca_entries(c, m, n, count, out);
  });
}

dmb_status dmb_aca_tree(dmb_ctx *c, int64_t *perm_out, double *centers_out) {
  return aca_guarded(c, [&] {
    const AcaState &A = c->aca;
    DMB_REQUIRE(A.valid, DMB_ERR_STATE, "no H-matrix operator built");
    if (perm_out)
      for (int64_t i = 0; i < A.n; i++) perm_out[i] = (int64_t)A.perm[i] + 1;
    if (centers_out) {
      DMB_CUDA(cudaMemcpyAsync(centers_out, c->d_centers.p, sizeof(double) * 3 * A.n, cudaMemcpyDeviceToHost,
                               c->stream));
      DMB_CUDA(cudaStreamSynchronize(c->stream));
    }
  });
}

dmb_status dmb_aca_lowrank(dmb_ctx *c, double k, double eta0, int quad_order, const int64_t *rows, int64_t m,
                           const int64_t *cols, int64_t n, double tol, int max_rank, int64_t max_output_bytes,
                           double *U_out, double *V_out, int64_t *rank_out) {
  return aca_guarded(c, [&] {
    DMB_REQUIRE(c->have_mesh && c->have_rwg, DMB_ERR_STATE, "mesh and RWG data must be uploaded first");
    DMB_REQUIRE(std::isfinite(tol) && tol > 0.0, DMB_ERR_ARGUMENT,
                "ACA tolerance must be finite and positive, got " + std::to_string(tol));
    DMB_REQUIRE(max_rank >= 1, DMB_ERR_ARGUMENT, "ACA max_rank must be at least 1, got " + std::to_string(max_rank));
    DMB_REQUIRE(std::isfinite(k) && k != 0.0 && std::isfinite(eta0) && eta0 != 0.0, DMB_ERR_ARGUMENT,
                "EFIE wavenumber and eta0 must be finite and nonzero");
    DMB_REQUIRE(m >= 1 && n >= 1 && rows && cols && U_out && V_out && rank_out, DMB_ERR_ARGUMENT,
                "bad ACA block arguments");
    const int64_t rmax = std::min<int64_t>(max_rank, std::min(m, n));
    const double planned = (double)rmax * (double)(m + n) * 16.0;
    DMB_REQUIRE(planned <= (double)max_output_bytes, DMB_ERR_ARGUMENT,
                "ACA low-rank factors require " + std::to_string((int64_t)planned) +
                    " bytes, exceeding max_output_bytes=" + std::to_string(max_output_bytes));
    std::vector<int> r(m), q(n);
    for (int64_t i = 0; i < m; i++) {
      DMB_REQUIRE(rows[i] >= 1 && rows[i] <= c->n, DMB_ERR_ARGUMENT, "row index out of range");
      r[i] = (int)(rows[i] - 1);
    }
    for (int64_t j = 0; j < n; j++) {
      DMB_REQUIRE(cols[j] >= 1 && cols[j] <= c->n, DMB_ERR_ARGUMENT, "column index out of range");
      q[j] = (int)(cols[j] - 1);
    }
    *rank_out = dmb::aca_lowrank_one(c, k, eta0, quad_order, r, q, tol, max_rank, U_out, V_out);
  });
}

dmb_status dmb_aca_nf_build(dmb_ctx *c, int kind, int precision, double *nnz_ratio_out) {
  return aca_guarded(c, [&] {
    dmb::aca_nf_build(c, kind, precision);
    if (nnz_ratio_out) *nnz_ratio_out = c->nnz_ratio;
  });
}

}  // extern "C"
