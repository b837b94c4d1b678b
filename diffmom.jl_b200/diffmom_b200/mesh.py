"""Triangle-surface meshes: the host-side ``TriMesh`` and its generators.

Mirrors DiffMoM.jl's L0/L1 layer for the meshes the EFIE path is run on:

* ``TriMesh`` -- ``src/Types.jl:123-126`` (xyz is 3 x Nv column-major in Julia,
  which is the same memory as the (Nv, 3) C-ordered array kept here; ``tri``
  holds 1-based vertex indices, (Nt, 3) C-ordered = Julia's 3 x Nt).
* ``make_rect_plate`` -- ``src/geometry/Mesh.jl:309-399``.
* ``make_circular_plate`` -- ``src/geometry/Mesh.jl:431-514``.
* ``make_icosphere`` -- the icosahedron subdivision of
  ``examples/04_pec_sphere_mie.jl:26-78`` / ``test/runtests.jl:373``.
* ``make_perturbed_ellipsoid`` -- seeded closed bodies for the learned
  preconditioner workload (no counterpart in the reference).

All generators are plain host code (O(Nt) integer/float work); the device
path starts at the C ABI upload.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class TriMesh:
    """Vertices ``xyz`` (Nv, 3) float64 and 1-based triangles ``tri`` (Nt, 3) int64."""

    xyz: np.ndarray
    tri: np.ndarray

    def __post_init__(self):
        self.xyz = np.ascontiguousarray(self.xyz, dtype=np.float64)
        self.tri = np.ascontiguousarray(self.tri, dtype=np.int64)
        if self.xyz.ndim != 2 or self.xyz.shape[1] != 3:
            raise ValueError("TriMesh.xyz must have shape (Nv, 3)")
        if self.tri.ndim != 2 or self.tri.shape[1] != 3:
            raise ValueError("TriMesh.tri must have shape (Nt, 3)")

    @property
    def nvertices(self) -> int:
        return self.xyz.shape[0]

    @property
    def ntriangles(self) -> int:
        return self.tri.shape[0]


def nvertices(mesh: TriMesh) -> int:
    return mesh.nvertices


def ntriangles(mesh: TriMesh) -> int:
    return mesh.ntriangles


def _positive_finite(name, value):
    v = float(value)
    if not (math.isfinite(v) and v > 0):
        raise ValueError(f"{name} must be finite and positive, got {value}")
    return v


def make_rect_plate(Lx, Ly, Nx: int, Ny: int) -> TriMesh:
    """Rectangular plate in z=0 centred at the origin, 2*Nx*Ny triangles.

    Vertex grid and split follow ``Mesh.jl:352-398``: coordinates
    ``half*(2*(i/cells)-1)`` with exact end points, cell (jx,jy) split into
    (v1,v2,v3) and (v1,v3,v4).
    """
    Lx = _positive_finite("Lx", Lx)
    Ly = _positive_finite("Ly", Ly)
    if Nx < 1 or Ny < 1:
        raise ValueError("Nx and Ny must be positive")
    hx, hy = Lx / 2, Ly / 2

    def axis(half, cells, i):
        if i == cells:
            return half
        if i == 0:
            return -half
        return half * (2 * (i / cells) - 1)

    xs = np.array([axis(hx, Nx, i) for i in range(Nx + 1)])
    ys = np.array([axis(hy, Ny, j) for j in range(Ny + 1)])
    X, Y = np.meshgrid(xs, ys)  # rows jy, cols jx
    xyz = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], axis=1)
    jy, jx = np.meshgrid(np.arange(Ny), np.arange(Nx), indexing="ij")
    jx = jx.ravel()
    jy = jy.ravel()
    v1 = jy * (Nx + 1) + jx + 1
    v2 = jy * (Nx + 1) + jx + 2
    v3 = (jy + 1) * (Nx + 1) + jx + 2
    v4 = (jy + 1) * (Nx + 1) + jx + 1
    tri = np.empty((2 * Nx * Ny, 3), dtype=np.int64)
    tri[0::2] = np.stack([v1, v2, v3], axis=1)
    tri[1::2] = np.stack([v1, v3, v4], axis=1)
    return TriMesh(xyz, tri)


def make_circular_plate(radius, Nr: int, Nphi: int) -> TriMesh:
    """Disk in z=0 with Nr rings of Nphi points (``Mesh.jl:431-514``).

    Nt = Nphi*(2*Nr-1), N_rwg = (3*Nt - Nphi)/2.
    """
    radius = _positive_finite("radius", radius)
    if Nr < 1 or Nphi < 3:
        raise ValueError("Nr >= 1 and Nphi >= 3 required")
    Nv = 1 + Nr * Nphi
    xyz = np.zeros((Nv, 3))
    idx = 1
    for ir in range(1, Nr + 1):
        r = radius * (ir / Nr)
        for ip in range(1, Nphi + 1):
            phi = 2 * math.pi * (ip - 1) / Nphi
            xyz[idx, 0] = r * math.cos(phi)
            xyz[idx, 1] = r * math.sin(phi)
            idx += 1
    tris = []
    for ip in range(1, Nphi + 1):
        v3 = 1 + ip + 1 if ip < Nphi else 2
        tris.append((1, 1 + ip, v3))
    for ir in range(1, Nr):
        off_in = 1 + (ir - 1) * Nphi
        off_out = 1 + ir * Nphi
        for ip in range(1, Nphi + 1):
            ipn = ip + 1 if ip < Nphi else 1
            a, b, c, d = off_in + ip, off_out + ip, off_out + ipn, off_in + ipn
            tris.append((a, b, c))
            tris.append((a, c, d))
    return TriMesh(xyz, np.array(tris, dtype=np.int64))


_ICO_VERTS = None


def make_icosphere(radius: float, subdivisions: int = 2) -> TriMesh:
    """Recursive icosahedron subdivision (``examples/04_pec_sphere_mie.jl:26-78``).

    Nt = 20*4^s; subdivisions=4 gives 5,120 triangles / 7,680 RWG.
    """
    phi = (1 + math.sqrt(5.0)) / 2
    verts0 = [(-1.0, phi, 0.0), (1.0, phi, 0.0), (-1.0, -phi, 0.0), (1.0, -phi, 0.0),
              (0.0, -1.0, phi), (0.0, 1.0, phi), (0.0, -1.0, -phi), (0.0, 1.0, -phi),
              (phi, 0.0, -1.0), (phi, 0.0, 1.0), (-phi, 0.0, -1.0), (-phi, 0.0, 1.0)]
    faces = [(1, 12, 6), (1, 6, 2), (1, 2, 8), (1, 8, 11), (1, 11, 12),
             (2, 6, 10), (6, 12, 5), (12, 11, 3), (11, 8, 7), (8, 2, 9),
             (4, 10, 5), (4, 5, 3), (4, 3, 7), (4, 7, 9), (4, 9, 10),
             (5, 10, 6), (3, 5, 12), (7, 3, 11), (9, 7, 8), (10, 9, 2)]
    verts = []
    for v in verts0:
        a = np.array(v)
        verts.append(a / math.sqrt(a @ a))
    for _ in range(subdivisions):
        edge_mid = {}
        new_faces = []

        def mid(i, j):
            key = (i, j) if i < j else (j, i)
            if key in edge_mid:
                return edge_mid[key]
            vm = (verts[i - 1] + verts[j - 1]) / 2
            vm = vm / math.sqrt(vm @ vm)
            verts.append(vm)
            edge_mid[key] = len(verts)
            return len(verts)

        for (i, j, k) in faces:
            a = mid(i, j)
            b = mid(j, k)
            c = mid(k, i)
            new_faces += [(i, a, c), (j, b, a), (k, c, b), (a, b, c)]
        faces = new_faces
    xyz = radius * np.array(verts)
    return TriMesh(xyz, np.array(faces, dtype=np.int64))


def make_geodesic_sphere(radius: float, frequency: int) -> TriMesh:
    """Icosahedron with every face split into frequency^2 triangles on a
    barycentric grid, projected onto the sphere: Nt = 20 f^2, N_rwg = 30 f^2
    (f = 18 gives 9,720 RWG; f = 24 gives 17,280)."""
    if frequency < 1:
        raise ValueError("frequency must be >= 1")
    base = make_icosphere(1.0, 0)
    V = base.xyz
    f = frequency
    keys = {}
    verts = []

    def vid(key, p):
        # key: the barycentric weights on the icosahedron's vertices, exact
        # integers, so points on shared edges/corners coincide across faces
        if key not in keys:
            keys[key] = len(verts) + 1
            verts.append(p / math.sqrt(p @ p))
        return keys[key]

    tris = []
    for a, b, c in base.tri - 1:
        A, B, C = V[a], V[b], V[c]
        grid = {}
        for i in range(f + 1):
            for j in range(f + 1 - i):
                w = f - i - j
                key = tuple(sorted((int(v), int(x)) for v, x in ((a, w), (b, i), (c, j)) if x))
                p = (A * w + B * i + C * j) / f
                grid[(i, j)] = vid(key, p)
        for i in range(f):
            for j in range(f - i):
                tris.append((grid[(i, j)], grid[(i + 1, j)], grid[(i, j + 1)]))
                if j + i + 1 < f:
                    tris.append((grid[(i + 1, j)], grid[(i + 1, j + 1)], grid[(i, j + 1)]))
    return TriMesh(radius * np.array(verts), np.array(tris, dtype=np.int64))


def _real_sph_harm(l, m, theta, phi):
    """Real spherical harmonic (unnormalised Legendre form) for perturbations."""
    from scipy.special import lpmv
    x = np.cos(theta)
    p = lpmv(abs(m), l, x)
    if m >= 0:
        return p * np.cos(m * phi)
    return p * np.sin(-m * phi)


def make_perturbed_ellipsoid(wavelength: float, seed: int, subdivisions: int = 4,
                             n_modes: int = 8, max_amplitude: float = 0.10,
                             frequency: int | None = None) -> TriMesh:
    """Seeded closed body: a sphere mesh mapped to an ellipsoid with semi-axes
    U[0.5,1.5] wavelengths, radially perturbed by ``n_modes`` random spherical
    harmonics with total relative amplitude <= ``max_amplitude``.

    The base mesh is the icosphere of ``subdivisions`` (4 gives 7,680 RWG), or
    the geodesic sphere of ``frequency`` when given (18 gives 9,720 RWG).
    """
    rng = np.random.default_rng(seed)
    base = make_geodesic_sphere(1.0, frequency) if frequency else make_icosphere(1.0, subdivisions)
    semi = rng.uniform(0.5, 1.5, size=3) * wavelength
    u = base.xyz
    theta = np.arccos(np.clip(u[:, 2], -1, 1))
    phi = np.arctan2(u[:, 1], u[:, 0])
    pert = np.zeros(u.shape[0])
    coefs = rng.uniform(-1, 1, size=n_modes)
    coefs *= max_amplitude / max(np.sum(np.abs(coefs)), 1e-12)
    for c in coefs:
        l = int(rng.integers(1, 6))
        m = int(rng.integers(-l, l + 1))
        y = _real_sph_harm(l, m, theta, phi)
        y = y / max(np.max(np.abs(y)), 1e-12)
        pert += c * y
    xyz = u * semi[None, :] * (1.0 + pert)[:, None]
    return TriMesh(xyz, base.tri.copy())


def triangle_area(mesh: TriMesh, t: int) -> float:
    """Area of triangle ``t`` (1-based), power-of-two scaled cross product
    as ``Mesh.jl:3205-3231``."""
    v = mesh.xyz[mesh.tri[t - 1] - 1]
    return float(_areas(v[None, 0], v[None, 1], v[None, 2])[0])


def _areas(a, b, c):
    e1 = b - a
    e2 = c - a
    s1 = np.max(np.abs(e1), axis=1)
    s2 = np.max(np.abs(e2), axis=1)
    _, x1 = np.frexp(s1)
    _, x2 = np.frexp(s2)
    a1 = np.ldexp(e1, -x1[:, None])
    b1 = np.ldexp(e2, -x2[:, None])
    cx = a1[:, 1] * b1[:, 2] - a1[:, 2] * b1[:, 1]
    cy = a1[:, 2] * b1[:, 0] - a1[:, 0] * b1[:, 2]
    cz = a1[:, 0] * b1[:, 1] - a1[:, 1] * b1[:, 0]
    cn = np.hypot(np.hypot(cx, cy), cz)
    fn, xn = np.frexp(cn)
    out = np.ldexp(0.5 * fn, xn + x1 + x2)
    out[cn == 0] = 0.0
    return out


def triangle_areas(mesh: TriMesh) -> np.ndarray:
    v = mesh.xyz[mesh.tri - 1]
    return _areas(v[:, 0], v[:, 1], v[:, 2])


def _two_sum(a, b):
    s = a + b
    bb = s - a
    return s, (a - (s - bb)) + (b - bb)


def triangle_centers(mesh: TriMesh) -> np.ndarray:
    """Centroids (``Mesh.jl:3161-3249``): error-free summation of the three
    coordinates, then one division by 3."""
    v = mesh.xyz[mesh.tri - 1]
    a, b, c = v[:, 0], v[:, 1], v[:, 2]
    s12, e12 = _two_sum(a, b)
    s123, e3 = _two_sum(s12, c)
    cl, ce = _two_sum(e12, e3)
    sl, se = _two_sum(s123, cl)
    return (sl + (se + ce)) / 3.0


def mesh_edge_max(mesh: TriMesh) -> float:
    v = mesh.xyz[mesh.tri - 1]
    e = np.concatenate([v[:, 1] - v[:, 0], v[:, 2] - v[:, 1], v[:, 0] - v[:, 2]])
    return float(np.max(np.linalg.norm(e, axis=1)))
