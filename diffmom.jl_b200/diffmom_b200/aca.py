"""H-matrix EFIE operator by adaptive cross approximation on the device.

Mirrors src/fast/ClusterTree.jl and src/fast/ACA.jl of DiffMoM.jl:
build_cluster_tree / is_admissible / leaf_nodes, aca_lowrank,
build_aca_operator -> ACAOperator (mul!, adjoint, getindex) and the
near-field preconditioner built from the operator's dense blocks
(src/solver/NearFieldPreconditioner.jl:952-1000).  Tree building and block
enumeration run in the library's host code; block fill, ACA and products on
the GPU.  Ranges are the reference's 1-based tree-order positions.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import _native as nat
from .mesh import TriMesh
from .rwg import RWGData

ETA0_DEFAULT = 376.730313668
_DEFAULT_MAX_ACA_BLOCK_TASKS = 2_000_000
_DEFAULT_MAX_ACA_STORAGE_BYTES = 2_000_000_000
_DEFAULT_MAX_ACA_GREEN_WORKSPACE_BYTES = 256 * 1024 * 1024
_DEFAULT_MAX_ACA_GREEN_CACHE_ENTRIES = 250_000
_DEFAULT_MAX_EFIE_CACHE_BYTES = 2_000_000_000
_DEFAULT_MAX_EFIE_ADJACENCY_PAIRS = 20_000_000
_QUAD_POINTS = {1: 1, 3: 3, 4: 4, 7: 7}


# ---------------------------------------------------------------------------
# cluster tree (src/fast/ClusterTree.jl)
# ---------------------------------------------------------------------------
@dataclass
class ClusterNode:
    """ClusterTree.jl:38-52: indices = 1-based tree-order positions;
    left / right = 1-based node ids (0 for a leaf)."""
    indices: range
    bbox_min: np.ndarray
    bbox_max: np.ndarray
    left: int
    right: int
    level: int


@dataclass
class ClusterTree:
    """ClusterTree.jl:54-66: nodes[0] is the root (node id 1); perm maps tree
    order to the original index (1-based), iperm the reverse."""
    nodes: list
    perm: np.ndarray
    iperm: np.ndarray
    leaf_size: int


def _plan(centers, leaf_size, eta=1.5, max_block_tasks=_DEFAULT_MAX_ACA_BLOCK_TASKS, want_tasks=False):
    lib = nat.load_library()
    c = np.ascontiguousarray(np.asarray(centers, dtype=np.float64).reshape(-1, 3))
    n = c.shape[0]
    perm = np.empty(max(n, 1), dtype=np.int64)
    nn = ctypes.c_int64()
    nt = ctypes.c_int64()
    nat.check_free(lib, lib.dmb_aca_plan(nat.dptr(c), n, int(leaf_size), float(eta), int(max_block_tasks),
                                         nat.lptr(perm), ctypes.byref(nn), None, None, ctypes.byref(nt), None, 0))
    nodes = np.empty((max(nn.value, 1), 5), dtype=np.int64)
    boxes = np.empty((max(nn.value, 1), 6), dtype=np.float64)
    tasks = np.empty((max(nt.value, 1), 5), dtype=np.int64) if want_tasks else None
    nat.check_free(lib, lib.dmb_aca_plan(nat.dptr(c), n, int(leaf_size), float(eta), int(max_block_tasks),
                                         nat.lptr(perm), ctypes.byref(nn), nat.lptr(nodes), nat.dptr(boxes),
                                         ctypes.byref(nt), nat.lptr(tasks) if want_tasks else None,
                                         nt.value if want_tasks else 0))
    return perm[:n], nodes[:nn.value], boxes[:nn.value], (tasks[:nt.value] if want_tasks else None)


_DEFAULT_MAX_CLUSTER_TREE_NODES = 30_000_000
_DEFAULT_MAX_CLUSTER_TREE_STORAGE_BYTES = 2_000_000_000
_CLUSTER_NODE_BYTES = 88  # UnitRange{Int} + two Vec3 + three Int


def cluster_tree_resource_bounds(N: int, leaf_size: int):
    """_cluster_tree_resource_bounds (ClusterTree.jl:13-36): the node count of
    a tree whose leaf count is the next power of two above ceil(N / leaf_size),
    and its storage (nodes plus perm, iperm and the centre order)."""
    target = -(-N // leaf_size)
    leaves = 1
    while leaves < target:
        leaves *= 2
    nodes = 2 * leaves - 1
    return nodes, nodes * _CLUSTER_NODE_BYTES + 3 * N * 8


def build_cluster_tree(centers, leaf_size: int = 64, max_nodes: int = _DEFAULT_MAX_CLUSTER_TREE_NODES,
                       max_storage_bytes: int = _DEFAULT_MAX_CLUSTER_TREE_STORAGE_BYTES) -> ClusterTree:
    """build_cluster_tree (ClusterTree.jl:82-166): median bisection along the
    longest bounding-box axis of `centers` (N x 3)."""
    c = np.asarray(centers, dtype=np.float64).reshape(-1, 3)
    if c.shape[0] == 0:
        raise ValueError("build_cluster_tree: centers must not be empty")
    if leaf_size < 1:
        raise ValueError(f"build_cluster_tree: leaf_size must be at least 1, got {leaf_size}")
    if max_nodes < 1 or max_storage_bytes < 1:
        raise ValueError("cluster-tree resource limits must be positive")
    nb, sb = cluster_tree_resource_bounds(c.shape[0], leaf_size)
    if nb > max_nodes:
        raise ValueError(f"cluster tree requires at most {nb} nodes, exceeding max_nodes={max_nodes}")
    if sb > max_storage_bytes:
        raise ValueError(f"cluster-tree arrays require {sb} bytes, exceeding max_storage_bytes={max_storage_bytes}")
    perm, nodes, boxes, _ = _plan(c, leaf_size, max_block_tasks=1 << 62)
    tree_nodes = [ClusterNode(range(int(r[0]), int(r[1]) + 1), b[:3].copy(), b[3:].copy(), int(r[2]), int(r[3]),
                              int(r[4])) for r, b in zip(nodes, boxes)]
    iperm = np.empty_like(perm)
    iperm[perm - 1] = np.arange(1, perm.size + 1)
    return ClusterTree(tree_nodes, perm, iperm, int(leaf_size))


def aca_block_tasks(centers, leaf_size: int = 64, eta: float = 1.5,
                    max_block_tasks: int = _DEFAULT_MAX_ACA_BLOCK_TASKS):
    """_enum_block_tasks! (ACA.jl:696-738): (row node id, column node id,
    kind) per task, kind "dense" or "lowrank", in the reference's order."""
    _, _, _, tasks = _plan(centers, leaf_size, eta, max_block_tasks, want_tasks=True)
    return [(int(t[0]), int(t[1]), "lowrank" if t[2] == 1 else "dense") for t in tasks]


def cluster_diameter(tree: ClusterTree, node_idx: int) -> float:
    nd = tree.nodes[node_idx - 1]
    span = nd.bbox_max - nd.bbox_min
    if not (np.all(np.isfinite(span)) and np.all(span >= 0)):
        raise ValueError(f"cluster {node_idx} has invalid bounding-box extents")
    return float(span.max())


def cluster_distance(tree: ClusterTree, i: int, j: int) -> float:
    a, b = tree.nodes[i - 1], tree.nodes[j - 1]
    g = np.maximum(np.maximum(a.bbox_min - b.bbox_max, b.bbox_min - a.bbox_max), 0.0)
    d = float(np.linalg.norm(g))
    if not math.isfinite(d):
        raise OverflowError("cluster distance overflowed")
    return d


def is_admissible(tree: ClusterTree, i: int, j: int, eta: float = 1.5) -> bool:
    """min(diam(i), diam(j)) <= eta dist(i, j) (ClusterTree.jl:216-246),
    decided exactly near the boundary."""
    lib = nat.load_library()
    a, b = tree.nodes[i - 1], tree.nodes[j - 1]
    bi = np.ascontiguousarray(np.concatenate([a.bbox_min, a.bbox_max]))
    bj = np.ascontiguousarray(np.concatenate([b.bbox_min, b.bbox_max]))
    out = ctypes.c_int()
    nat.check_free(lib, lib.dmb_aca_admissible(nat.dptr(bi), nat.dptr(bj), float(eta), ctypes.byref(out)))
    return bool(out.value)


def is_leaf(tree: ClusterTree, node_idx: int) -> bool:
    return tree.nodes[node_idx - 1].left == 0


def leaf_nodes(tree: ClusterTree) -> list:
    return [i + 1 for i, nd in enumerate(tree.nodes) if nd.left == 0]


# ---------------------------------------------------------------------------
# EFIE entry cache and aca_lowrank
# ---------------------------------------------------------------------------
@dataclass
class EFIECache:
    """What _build_efie_cache (EFIE.jl:332-398) holds for entry evaluation: the
    device keeps the triangle cache; k, quad_order and eta0 select the entries."""
    device: object
    k: float
    quad_order: int = 3
    eta0: float = ETA0_DEFAULT


def build_efie_cache(mesh: TriMesh, rwg: RWGData, k, quad_order: int = 3, eta0: float = ETA0_DEFAULT,
                     device=None) -> EFIECache:
    from .api import EFIEDevice
    if quad_order not in _QUAD_POINTS:
        raise ValueError(f"Unsupported quadrature order {quad_order}. Use 1, 3, 4, or 7.")
    return EFIECache(device or EFIEDevice(mesh, rwg), float(k), int(quad_order), float(eta0))


def efie_cache_with_prefactor_scale(cache: EFIECache, k, scale: float) -> EFIECache:
    """The entries of `cache` at wavenumber k with every prefactor multiplied
    by `scale` (the reference test's _efie_cache_with_prefactors)."""
    return EFIECache(cache.device, float(k), cache.quad_order, cache.eta0 * float(scale))


def aca_lowrank(cache: EFIECache, row_indices, col_indices, tol: float = 1e-6, max_rank: int = 50,
                max_output_bytes: int = _DEFAULT_MAX_ACA_STORAGE_BYTES):
    """aca_lowrank (ACA.jl:351-554): partially pivoted ACA of the EFIE block
    Z[rows, cols] (1-based index lists) on the device; returns (U, V) with
    block ~= U V^H."""
    rows = np.ascontiguousarray(row_indices, dtype=np.int64)
    cols = np.ascontiguousarray(col_indices, dtype=np.int64)
    m, n = rows.size, cols.size
    if not (math.isfinite(tol) and tol > 0):
        raise ValueError(f"ACA tolerance must be finite and positive, got {tol}")
    if max_rank < 1:
        raise ValueError(f"ACA max_rank must be at least 1, got {max_rank}")
    r = max(1, min(max_rank, m, n))
    U = np.zeros((m, r), dtype=np.complex128, order="F")
    V = np.zeros((n, r), dtype=np.complex128, order="F")
    rank = ctypes.c_int64()
    cache.device.ctx.call("dmb_aca_lowrank", cache.k, cache.eta0, cache.quad_order, nat.lptr(rows), m,
                          nat.lptr(cols), n, float(tol), int(max_rank), int(max_output_bytes), nat.dptr(U),
                          nat.dptr(V), ctypes.byref(rank))
    return U[:, :rank.value].copy(), V[:, :rank.value].copy()


# ---------------------------------------------------------------------------
# the operator
# ---------------------------------------------------------------------------
@dataclass
class DenseBlock:
    """ACA.jl:97-108: a near (inadmissible) block; ranges are 1-based tree
    order."""
    row_range: range
    col_range: range
    op: "ACAOperator" = field(repr=False, default=None)
    index: int = -1
    fallback: bool = False

    @property
    def data(self) -> np.ndarray:
        return self.op._block_data(self.index)[0]


@dataclass
class LowRankBlock:
    """ACA.jl:110-121: a far block as U V^H (U m x r, V n x r)."""
    row_range: range
    col_range: range
    rank: int
    op: "ACAOperator" = field(repr=False, default=None)
    index: int = -1

    @property
    def U(self) -> np.ndarray:
        return self.op._block_data(self.index)[0]

    @property
    def V(self) -> np.ndarray:
        return self.op._block_data(self.index)[1]


def _scaled(Ax: np.ndarray, alpha, beta, y):
    alpha, beta = complex(alpha), complex(beta)
    if y is None:
        out = Ax if alpha == 1 else alpha * Ax
        return out
    if y.shape != Ax.shape:
        raise ValueError(f"output has shape {y.shape}, expected {Ax.shape}")
    with np.errstate(over="ignore", invalid="ignore"):
        if beta == 0:
            y[...] = alpha * Ax
        else:
            y[...] = alpha * Ax + beta * y
    if not np.all(np.isfinite(y)):
        raise OverflowError("ACA scaled product is outside the representable ComplexF64 range")
    return y


class ACAOperator:
    """H-matrix operator (ACA.jl:173-181) resident on a device context."""

    def __init__(self, device, info: nat.AcaInfo, k: float, eta0: float, quad_order: int,
                 owns_device: bool = False):
        self.device = device
        self._owns_device = owns_device
        # a device context holds one H-matrix: a later build on it replaces
        # this operator's data, after which this object refuses to run
        device._aca_current = self
        self.N = device.N
        self.shape = (self.N, self.N)
        self.k, self.eta0, self.quad_order = k, eta0, quad_order
        self.info = {f: getattr(info, f) for f, _ in nat.AcaInfo._fields_}
        B = np.empty((max(1, info.n_dense + info.n_lowrank), 7), dtype=np.int64)
        device.ctx.call("dmb_aca_blocks", nat.lptr(B))
        self._blocks = B[:info.n_dense + info.n_lowrank]
        self._cache = {}
        self.dense_blocks, self.lowrank_blocks = [], []
        for i, b in enumerate(self._blocks):
            rr, cr = range(int(b[1]), int(b[2]) + 1), range(int(b[3]), int(b[4]) + 1)
            if b[0] == 0:
                self.dense_blocks.append(DenseBlock(rr, cr, self, i, bool(b[6])))
            else:
                self.lowrank_blocks.append(LowRankBlock(rr, cr, int(b[5]), self, i))
        perm = np.empty(self.N, dtype=np.int64)
        device.ctx.call("dmb_aca_tree", nat.lptr(perm), None)
        iperm = np.empty_like(perm)
        iperm[perm - 1] = np.arange(1, self.N + 1)
        self.perm, self.iperm = perm, iperm

    def _check_current(self):
        if getattr(self.device, "_aca_current", None) is not self:
            raise nat.DiffMoMError("this H-matrix operator was replaced by a later build_aca_operator "
                                   "on the same device")

    def _select(self):
        self._check_current()
        self.device.ctx.call("dmb_set_option", nat.OPT_OPERATOR, 1)

    def _block_data(self, i):
        if i not in self._cache:
            self._check_current()
            b = self._blocks[i]
            m, n = int(b[2] - b[1] + 1), int(b[4] - b[3] + 1)
            if b[0] == 0:
                a = np.empty((m, n), dtype=np.complex128, order="F")
                self.device.ctx.call("dmb_aca_block_data", i, nat.dptr(a), None)
                self._cache[i] = (a, None)
            else:
                r = int(b[5])
                U = np.empty((m, r), dtype=np.complex128, order="F")
                V = np.empty((n, r), dtype=np.complex128, order="F")
                self.device.ctx.call("dmb_aca_block_data", i, nat.dptr(U), nat.dptr(V))
                self._cache[i] = (U, V)
        return self._cache[i]

    def matvec(self, x, mode: int = 0) -> np.ndarray:
        """mode 0: A x, 1: A^H x, 2: A^T x (x: N or N x R)."""
        self._check_current()
        X = nat.c128(x)
        nrhs = 1 if X.ndim == 1 else X.shape[1]
        Y = np.empty_like(X)
        self.device.ctx.call("dmb_aca_matvec", nat.dptr(X), nat.dptr(Y), nrhs, int(mode))
        return Y

    def __matmul__(self, x):
        return self.matvec(x, 0)

    def mul(self, x, alpha=1.0, beta=0.0, y=None):
        """mul!(y, A, x, alpha, beta) (ACA.jl:1130-1221): alpha A x + beta y;
        y is overwritten when given, beta = 0 ignores its contents."""
        return _scaled(self.matvec(x, 0), alpha, beta, y)

    def adjoint(self) -> "ACAAdjointOperator":
        return ACAAdjointOperator(self)

    @property
    def H(self) -> "ACAAdjointOperator":
        return self.adjoint()

    def entries(self, m, n) -> np.ndarray:
        """getindex (ACA.jl:220-222): EFIE entries Z[m, n] (1-based)."""
        self._check_current()
        m = np.ascontiguousarray(np.atleast_1d(m), dtype=np.int64)
        n = np.ascontiguousarray(np.atleast_1d(n), dtype=np.int64)
        out = np.empty(m.size, dtype=np.complex128)
        self.device.ctx.call("dmb_aca_entries", nat.lptr(m), nat.lptr(n), m.size, nat.dptr(out))
        return out

    def __getitem__(self, ij):
        i, j = ij
        return complex(self.entries([i + 1], [j + 1])[0])

    def to_dense(self) -> np.ndarray:
        """The approximated matrix in the original order (tests and small N)."""
        P = np.zeros((self.N, self.N), dtype=np.complex128)
        p = self.perm - 1
        for b in self.dense_blocks:
            P[np.ix_(p[b.row_range.start - 1:b.row_range.stop - 1], p[b.col_range.start - 1:b.col_range.stop - 1])] = b.data
        for b in self.lowrank_blocks:
            if b.rank:
                P[np.ix_(p[b.row_range.start - 1:b.row_range.stop - 1],
                         p[b.col_range.start - 1:b.col_range.stop - 1])] = b.U @ b.V.conj().T
        return P

    def build_nearfield(self, factorization: str = "lu", precision: str = "fp64"):
        from .api import NearFieldPreconditionerData, _PRECISIONS
        kinds = {"lu": nat.PRECOND_NF_LU, "diag": nat.PRECOND_NF_DIAG}
        if factorization not in kinds:
            raise ValueError(f"invalid factorization={factorization}; expected one of (:lu, :diag)")
        if precision not in _PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}")
        self._select()
        ratio = ctypes.c_double()
        self.device.ctx.call("dmb_aca_nf_build", kinds[factorization], _PRECISIONS[precision], ctypes.byref(ratio))
        P = NearFieldPreconditionerData(self.device, kinds[factorization], math.inf, ratio.value)
        self.device.preconditioner = P
        return P

    def gmres(self, rhs, tol=1e-8, maxiter=200, preconditioner=None, precond_side="left",
              check_gmres_convergence=True, adjoint=False):
        self._select()
        return self.device.gmres(rhs, tol=tol, maxiter=maxiter, preconditioner=preconditioner,
                                 precond_side=precond_side, check_gmres_convergence=check_gmres_convergence,
                                 adjoint=adjoint)

    def close(self):
        """Release the device context if build_aca_operator created it (a
        context passed in by the caller stays open)."""
        if self._owns_device:
            self.device.close()


class ACAAdjointOperator:
    """ACA.jl:210-218: y = A^H x."""

    def __init__(self, op: ACAOperator):
        self.op = op
        self.shape = op.shape

    def __matmul__(self, x):
        return self.op.matvec(x, 1)

    def mul(self, x, alpha=1.0, beta=0.0, y=None):
        """mul!(y, A', x, alpha, beta) (ACA.jl:1231-1323)."""
        return _scaled(self.op.matvec(x, 1), alpha, beta, y)

    def __getitem__(self, ij):
        i, j = ij
        return complex(np.conj(self.op.entries([j + 1], [i + 1])[0]))


def build_aca_operator(mesh: TriMesh, rwg: RWGData, k, leaf_size: int = 64, eta: float = 1.5,
                       aca_tol: float = 1e-6, max_rank: int = 50, quad_order: int = 3,
                       eta0: float = ETA0_DEFAULT, mesh_precheck: bool = True, allow_boundary: bool = True,
                       require_closed: bool = False, area_tol_rel: float = 1e-12,
                       max_block_tasks: int = _DEFAULT_MAX_ACA_BLOCK_TASKS,
                       max_storage_bytes: int = _DEFAULT_MAX_ACA_STORAGE_BYTES,
                       max_cache_bytes: int = _DEFAULT_MAX_EFIE_CACHE_BYTES,
                       max_adjacency_pairs: int = _DEFAULT_MAX_EFIE_ADJACENCY_PAIRS,
                       max_green_cache_bytes: int = _DEFAULT_MAX_ACA_GREEN_WORKSPACE_BYTES,
                       max_green_cache_entries: int = _DEFAULT_MAX_ACA_GREEN_CACHE_ENTRIES,
                       device=None) -> ACAOperator:
    """build_aca_operator (ACA.jl:802-1103) on the GPU.

    The device evaluates entries on the fly and keeps no Green-matrix cache;
    max_green_cache_* and max_cache_bytes are validated as the reference does
    (one quadrature-pair Green matrix and the triangle cache must fit)."""
    from .api import EFIEDevice
    if not (math.isfinite(aca_tol) and aca_tol > 0):
        raise ValueError(f"ACA tolerance must be finite and positive, got {aca_tol}")
    if max_rank < 1:
        raise ValueError(f"ACA max_rank must be at least 1, got {max_rank}")
    if leaf_size < 1:
        raise ValueError(f"ACA leaf_size must be at least 1, got {leaf_size}")
    if not (math.isfinite(eta) and eta > 0):
        raise ValueError(f"ACA eta must be finite and positive, got {eta}")
    if max_block_tasks < 1:
        raise ValueError(f"max_block_tasks must be positive, got {max_block_tasks}")
    if max_storage_bytes < 1:
        raise ValueError(f"max_storage_bytes must be positive, got {max_storage_bytes}")
    if max_green_cache_bytes < 1:
        raise ValueError(f"max_green_cache_bytes must be positive, got {max_green_cache_bytes}")
    if max_green_cache_entries < 0:
        raise ValueError(f"max_green_cache_entries must be nonnegative, got {max_green_cache_entries}")
    if max_adjacency_pairs < 1:
        raise ValueError(f"max_adjacency_pairs must be positive, got {max_adjacency_pairs}")
    if quad_order not in _QUAD_POINTS:
        raise ValueError(f"Unsupported quadrature order {quad_order}. Use 1, 3, 4, or 7.")
    nq = _QUAD_POINTS[quad_order]
    if 16 * nq * nq > max_green_cache_bytes:
        raise ValueError(f"one ACA Green matrix requires {16 * nq * nq} raw bytes, exceeding "
                         f"max_green_cache_bytes={max_green_cache_bytes}")
    # the per-triangle cache: quadrature points, weights and basis data
    cache_bytes = mesh.ntriangles * 8 * (9 + 3 + 1 + 14 + 63 + 18)
    if cache_bytes > max_cache_bytes:
        raise ValueError(f"EFIE cache requires {cache_bytes} bytes, exceeding max_cache_bytes={max_cache_bytes}")
    if rwg.mesh is not mesh:
        raise ValueError("RWG data was built for a different mesh")
    dev = device or EFIEDevice(mesh, rwg)
    info = nat.AcaInfo()
    try:
        dev.ctx.call("dmb_aca_build", float(k), float(eta0), int(quad_order), int(leaf_size), float(eta),
                     float(aca_tol), int(max_rank), int(max_block_tasks), int(max_storage_bytes), ctypes.byref(info))
    except Exception:
        if device is None:
            dev.close()
        raise
    dev.preconditioner = None
    return ACAOperator(dev, info, float(k), float(eta0), int(quad_order), owns_device=device is None)
