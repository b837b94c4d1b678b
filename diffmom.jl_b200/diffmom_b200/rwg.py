"""RWG basis data (``src/Types.jl:138-152``, ``src/basis/RWG.jl:102-143``).

``build_rwg`` creates one basis function per interior edge (an edge shared by
exactly two triangles).  T+ is the lower-indexed triangle (the one that first
registered the edge, ``RWG.jl:7-19``); ``evert`` is the sorted vertex pair.

Ordering: the reference enumerates a ``Dict`` whose iteration order cannot be
reproduced outside Julia, so this mirror uses the canonical sorted-edge-key
order.  Every consumer (the oracle and the device library) takes the RWG
arrays as given, so any order -- including Julia's -- is accepted across the
C ABI.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .mesh import TriMesh, triangle_areas


@dataclass
class RWGData:
    mesh: TriMesh
    nedges: int
    tplus: np.ndarray       # (N,) int64, 1-based
    tminus: np.ndarray      # (N,) int64, 1-based
    evert: np.ndarray       # (N, 2) int64, 1-based (Julia 2 x N column-major)
    vplus_opp: np.ndarray   # (N,) int64, 1-based
    vminus_opp: np.ndarray  # (N,) int64, 1-based
    len: np.ndarray         # (N,) float64
    area_plus: np.ndarray   # (N,) float64
    area_minus: np.ndarray  # (N,) float64
    coeff_plus: np.ndarray  # (N,) float64 (all 1.0)
    coeff_minus: np.ndarray
    has_periodic_bloch: bool = False

    def arrays(self):
        return dict(tplus=self.tplus, tminus=self.tminus, evert=self.evert,
                    vplus_opp=self.vplus_opp, vminus_opp=self.vminus_opp,
                    len=self.len, area_plus=self.area_plus, area_minus=self.area_minus)


def build_rwg(mesh: TriMesh, precheck: bool = True) -> RWGData:
    tri = mesh.tri
    Nt = tri.shape[0]
    if precheck:
        if Nt == 0:
            raise ValueError("build_rwg: mesh has no triangles")
        if tri.min() < 1 or tri.max() > mesh.nvertices:
            raise ValueError("build_rwg: triangle vertex index out of range")
        areas = triangle_areas(mesh)
        if np.any(~np.isfinite(areas)) or np.any(areas <= 0):
            raise ValueError("build_rwg: degenerate triangle")
    # edge le of triangle t joins tri[t, le] and tri[t, (le+1)%3]; opposite tri[t, (le+2)%3]
    a = tri[:, [0, 1, 2]].ravel()
    b = tri[:, [1, 2, 0]].ravel()
    opp = tri[:, [2, 0, 1]].ravel()
    tids = np.repeat(np.arange(1, Nt + 1, dtype=np.int64), 3)
    lo = np.minimum(a, b)
    hi = np.maximum(a, b)
    order = np.lexsort((tids, hi, lo))
    lo, hi, opp, tids = lo[order], hi[order], opp[order], tids[order]
    key_change = np.ones(lo.size, dtype=bool)
    key_change[1:] = (lo[1:] != lo[:-1]) | (hi[1:] != hi[:-1])
    starts = np.flatnonzero(key_change)
    counts = np.diff(np.append(starts, lo.size))
    sel = starts[counts == 2]
    tp = tids[sel]
    tm = tids[sel + 1]
    vpo = opp[sel]
    vmo = opp[sel + 1]
    ev = np.stack([lo[sel], hi[sel]], axis=1)
    r1 = mesh.xyz[ev[:, 0] - 1]
    r2 = mesh.xyz[ev[:, 1] - 1]
    d = r2 - r1
    ln = np.hypot(np.hypot(d[:, 0], d[:, 1]), d[:, 2])
    if np.any(~(ln > 0)):
        raise ValueError("RWG edge has zero or unrepresentable length")
    areas = triangle_areas(mesh)
    N = tp.size
    return RWGData(mesh=mesh, nedges=N, tplus=tp, tminus=tm,
                   evert=np.ascontiguousarray(ev), vplus_opp=vpo, vminus_opp=vmo,
                   len=ln, area_plus=areas[tp - 1].copy(), area_minus=areas[tm - 1].copy(),
                   coeff_plus=np.ones(N), coeff_minus=np.ones(N))


def rwg_centers(mesh: TriMesh, rwg: RWGData) -> np.ndarray:
    """Mean of the two supporting centroids (``NearFieldPreconditioner.jl:247-257``)."""
    from .mesh import triangle_centers
    cen = triangle_centers(mesh)
    a = cen[rwg.tplus - 1]
    b = cen[rwg.tminus - 1]
    # Mesh.jl:3492-3507 _safe_midpoint_component: canonical order, then
    # lower + (upper-lower)/2 for equal signs, (lower+upper)/2 otherwise.
    lower = np.minimum(a, b)
    upper = np.maximum(a, b)
    same = np.signbit(lower) == np.signbit(upper)
    return np.where(same, lower + (upper - lower) / 2, (lower + upper) / 2)


def basis_triangles(rwg: RWGData, n: int):
    return int(rwg.tplus[n - 1]), int(rwg.tminus[n - 1])
