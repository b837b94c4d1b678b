"""CPU restatement of DiffMoM.jl's H-matrix (ACA) operator.

TEST INFRASTRUCTURE ONLY: this module is the checker of diffmom_b200's
dmb_aca_* entry points.  Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg may import it; the library never does.

Restates, in plain Python (exact rationals where the reference uses them):
  build_cluster_tree        src/fast/ClusterTree.jl:82-166
  cluster_diameter          src/fast/ClusterTree.jl:168-180
  cluster_distance          src/fast/ClusterTree.jl:182-191 (float path)
  is_admissible             src/fast/ClusterTree.jl:216-246 (+ :193-214 exact)
  enum_block_tasks          src/fast/ACA.jl:696-738
  aca_lowrank               src/fast/ACA.jl:351-554 (entries from a dense block)
  hmatrix_matvec            src/fast/ACA.jl:1130-1221 / 1231-1323
Indices here are 0-based; node ranges are inclusive (lo, hi) like the
reference's UnitRange.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from fractions import Fraction

import numpy as np


@dataclass
class Node:
    lo: int
    hi: int
    bmin: tuple
    bmax: tuple
    left: int = -1
    right: int = -1
    level: int = 0


@dataclass
class Tree:
    nodes: list
    perm: list
    leaf_size: int


def _isless_key(v: float):
    # Julia's isless on finite doubles: -0.0 sorts before 0.0
    return (v, 0 if math.copysign(1.0, v) < 0 else 1)


def build_cluster_tree(centers, leaf_size: int = 64) -> Tree:
    """ClusterTree.jl:82-166: recursive median bisection along the longest
    bounding-box axis with a stable sort (Julia >= 1.9 default)."""
    c = np.asarray(centers, dtype=np.float64).reshape(-1, 3)
    n = c.shape[0]
    if n == 0:
        raise ValueError("build_cluster_tree: centers must not be empty")
    if leaf_size < 1:
        raise ValueError(f"build_cluster_tree: leaf_size must be at least 1, got {leaf_size}")
    if not np.all(np.isfinite(c)):
        raise ValueError("build_cluster_tree: centers must be finite")
    pts = [tuple(float(x) for x in row) for row in c]
    perm = list(range(n))
    nodes: list[Node] = []

    def build(lo: int, hi: int, level: int) -> int:
        bmin = [math.inf] * 3
        bmax = [-math.inf] * 3
        for k in range(lo, hi + 1):
            p = pts[perm[k]]
            for a in range(3):
                bmin[a] = min(bmin[a], p[a])
                bmax[a] = max(bmax[a], p[a])
        span = [bmax[a] - bmin[a] for a in range(3)]
        if hi - lo + 1 <= leaf_size:
            nodes.append(Node(lo, hi, tuple(bmin), tuple(bmax), -1, -1, level))
            return len(nodes) - 1
        axis = 0
        if span[1] > span[axis]:
            axis = 1
        if span[2] > span[axis]:
            axis = 2
        perm[lo:hi + 1] = sorted(perm[lo:hi + 1], key=lambda k: _isless_key(pts[k][axis]))
        mid = ((lo + 1 + hi + 1) >> 1) - 1  # (lo + hi) >> 1 on 1-based positions
        nodes.append(Node(lo, hi, tuple(bmin), tuple(bmax), -1, -1, level))
        me = len(nodes) - 1
        left = build(lo, mid, level + 1)
        right = build(mid + 1, hi, level + 1)
        nodes[me].left = left
        nodes[me].right = right
        return me

    build(0, n - 1, 0)
    return Tree(nodes, perm, leaf_size)


def cluster_diameter(tree: Tree, i: int) -> float:
    nd = tree.nodes[i]
    return max(nd.bmax[a] - nd.bmin[a] for a in range(3))


def _admissible_exact(a: Node, b: Node, eta: float) -> bool:
    """ClusterTree.jl:193-214: the whole comparison in exact rationals."""
    gaps = [max(Fraction(a.bmin[c]) - Fraction(b.bmax[c]), Fraction(b.bmin[c]) - Fraction(a.bmax[c]), Fraction(0))
            for c in range(3)]
    si = max(Fraction(a.bmax[c]) - Fraction(a.bmin[c]) for c in range(3))
    sj = max(Fraction(b.bmax[c]) - Fraction(b.bmin[c]) for c in range(3))
    diam = min(si, sj)
    e = Fraction(eta)
    return diam * diam <= e * e * (gaps[0] ** 2 + gaps[1] ** 2 + gaps[2] ** 2)


def _ulp_above(x: float) -> float:
    x = abs(x)
    return math.nextafter(x, math.inf) - x


def box_admissible(a: Node, b: Node, eta: float) -> bool:
    """is_admissible (ClusterTree.jl:223-246)."""
    if not (math.isfinite(eta) and eta > 0):
        raise ValueError(f"eta must be finite and positive, got {eta}")
    g = [max(a.bmin[c] - b.bmax[c], b.bmin[c] - a.bmax[c], 0.0) for c in range(3)]
    d = math.hypot(g[0], g[1], g[2])
    if d <= 0.0:
        return False
    diam = min(max(a.bmax[c] - a.bmin[c] for c in range(3)), max(b.bmax[c] - b.bmin[c] for c in range(3)))
    sd = eta * d
    if math.isinf(sd):
        return True
    if sd == 0.0:
        return diam == 0.0
    unc = 64 * _ulp_above(max(diam, sd))
    if math.isfinite(unc) and abs(diam - sd) > unc:
        return diam <= sd
    return _admissible_exact(a, b, eta)


def is_admissible(tree: Tree, i: int, j: int, eta: float = 1.5) -> bool:
    return box_admissible(tree.nodes[i], tree.nodes[j], eta)


def enum_block_tasks(tree: Tree, eta: float = 1.5, max_block_tasks: int = 2_000_000):
    """_enum_block_tasks! (ACA.jl:696-738): list of (row node, col node, kind)
    with kind 0 = dense, 1 = low-rank, in the reference's recursion order."""
    tasks = []

    def rec(rn: int, cn: int):
        if len(tasks) >= max_block_tasks:
            raise ValueError(f"ACA block enumeration exceeds max_block_tasks={max_block_tasks}")
        if is_admissible(tree, rn, cn, eta):
            tasks.append((rn, cn, 1))
            return
        r, c = tree.nodes[rn], tree.nodes[cn]
        rl, cl = r.left < 0, c.left < 0
        if rl and cl:
            tasks.append((rn, cn, 0))
            return
        if rl:
            rec(rn, c.left)
            rec(rn, c.right)
        elif cl:
            rec(r.left, cn)
            rec(r.right, cn)
        else:
            rec(r.left, c.left)
            rec(r.left, c.right)
            rec(r.right, c.left)
            rec(r.right, c.right)

    rec(0, 0)
    return tasks


# --- aca_lowrank: scaled magnitudes (ACA.jl:232-306) -------------------------
def _vec_norm(v: np.ndarray):
    scale = float(max(np.max(np.abs(v.real)), np.max(np.abs(v.imag))))
    if not scale > 0.0:
        raise OverflowError("ACA low-rank update has zero norm")
    sn = math.sqrt(float(np.sum((v.real / scale) ** 2 + (v.imag / scale) ** 2)))
    sf, se = math.frexp(scale)
    nf, ne = math.frexp(sf * sn)
    return scale, sn, (nf, se + ne)


def _mag_mul(a, b):
    f, e = math.frexp(a[0] * b[0])
    return (f, a[1] + b[1] + e)


def _mag_less(a, b):
    return a[0] < b[0] if a[1] == b[1] else a[1] < b[1]


def _mag_ratio(a, b):
    return math.ldexp(a[0] / b[0], a[1] - b[1])


def aca_lowrank(block: np.ndarray, tol: float = 1e-6, max_rank: int = 50):
    """aca_lowrank (ACA.jl:351-554) with the entries taken from `block`
    (m x n).  Returns (U, V, converged) with block ~= U V^H."""
    if not (math.isfinite(tol) and tol > 0):
        raise ValueError(f"ACA tolerance must be finite and positive, got {tol}")
    if max_rank < 1:
        raise ValueError(f"ACA max_rank must be at least 1, got {max_rank}")
    Z = np.asarray(block, dtype=np.complex128)
    m, n = Z.shape
    max_rank = min(max_rank, m, n)
    U_cols, V_cols, U_n, V_n, T_n = [], [], [], [], []
    used_r = np.zeros(m, bool)
    used_c = np.zeros(n, bool)
    frob_scale = None
    fsq = 0.0
    prow = 0
    converged = False
    for _ in range(max_rank):
        row = Z[prow, :].copy()
        for u, v in zip(U_cols, V_cols):
            row -= u[prow] * np.conj(v)
        av = np.abs(row)
        pc, best = -1, 0.0
        for jj in range(n):
            if av[jj] > best and not used_c[jj]:
                best, pc = av[jj], jj
        if pc < 0 or best == 0.0:
            free = np.flatnonzero(~used_c)
            if free.size == 0:
                break
            pc = int(free[0])
            if abs(row[pc]) == 0.0:
                break
        piv = row[pc]
        col = Z[:, pc].copy()
        for u, v in zip(U_cols, V_cols):
            col -= u * np.conj(v[pc])
        uk = col / piv
        vk = np.conj(row)
        if not (np.all(np.isfinite(uk)) and np.all(np.isfinite(vk))):
            raise OverflowError("ACA low-rank update became non-finite")
        un, vn = _vec_norm(uk), _vec_norm(vk)
        term = _mag_mul(un[2], vn[2])
        U_cols.append(uk)
        V_cols.append(vk)
        U_n.append(un)
        V_n.append(vn)
        T_n.append(term)
        used_r[prow] = True
        used_c[pc] = True
        if frob_scale is None:
            frob_scale = term
        elif _mag_less(frob_scale, term):
            r = _mag_ratio(frob_scale, term)
            fsq *= r * r
            frob_scale = term
        tr = _mag_ratio(term, frob_scale)
        cross = 0.0
        for p in range(len(U_cols) - 1):
            pr = _mag_ratio(T_n[p], frob_scale)
            uc = np.vdot(U_cols[p] / U_n[p][0], uk / un[0]) / (U_n[p][1] * un[1])
            vc = np.vdot(V_cols[p] / V_n[p][0], vk / vn[0]) / (V_n[p][1] * vn[1])
            cross += 2.0 * pr * tr * (uc * np.conj(vc)).real
        fsq = max(fsq + tr * tr + cross, 0.0)
        if tr < tol * math.sqrt(fsq):
            converged = True
            break
        au = np.abs(uk)
        nxt, bu = -1, 0.0
        for ii in range(m):
            if not used_r[ii] and au[ii] > bu:
                bu, nxt = au[ii], ii
        if nxt < 0:
            break
        prow = nxt
    r = len(U_cols)
    U = np.stack(U_cols, 1) if r else np.zeros((m, 0), complex)
    V = np.stack(V_cols, 1) if r else np.zeros((n, 0), complex)
    return U, V, converged


@dataclass
class Block:
    kind: int           # 0 dense, 1 low-rank
    r0: int
    m: int
    c0: int
    n: int
    data: np.ndarray = None
    U: np.ndarray = None
    V: np.ndarray = None
    converged: bool = True


def build_hmatrix(Z: np.ndarray, centers, leaf_size=64, eta=1.5, aca_tol=1e-6, max_rank=50):
    """build_aca_operator (ACA.jl:802-1103) from a dense Z: tree, tasks,
    dense blocks and ACA blocks, in task order."""
    tree = build_cluster_tree(centers, leaf_size)
    tasks = enum_block_tasks(tree, eta)
    perm = np.asarray(tree.perm)
    blocks = []
    for rn, cn, kind in tasks:
        r, c = tree.nodes[rn], tree.nodes[cn]
        rows, cols = perm[r.lo:r.hi + 1], perm[c.lo:c.hi + 1]
        sub = Z[np.ix_(rows, cols)]
        b = Block(kind, r.lo, r.hi - r.lo + 1, c.lo, c.hi - c.lo + 1)
        if kind == 0:
            b.data = sub.copy()
        else:
            try:
                b.U, b.V, b.converged = aca_lowrank(sub, aca_tol, max_rank)
            except OverflowError as e:
                if "non-finite" not in str(e):
                    raise
                b.kind, b.data = 0, sub.copy()
        blocks.append(b)
    return tree, tasks, blocks


def hmatrix_matvec(blocks, perm, x: np.ndarray, mode: int = 0) -> np.ndarray:
    """y = A x (mode 0), A^H x (1) or A^T x (2) of an H-matrix given in tree
    order; x, y in the original order."""
    perm = np.asarray(perm)
    xp = np.asarray(x, dtype=np.complex128)[perm]
    yp = np.zeros_like(xp)
    for b in blocks:
        rs, cs = slice(b.r0, b.r0 + b.m), slice(b.c0, b.c0 + b.n)
        if b.kind == 0:
            A = b.data
        else:
            A = b.U @ b.V.conj().T
        if mode == 0:
            yp[rs] += A @ xp[cs]
        elif mode == 1:
            yp[cs] += A.conj().T @ xp[rs]
        else:
            yp[cs] += A.T @ xp[rs]
    y = np.empty_like(yp)
    y[perm] = yp
    return y
