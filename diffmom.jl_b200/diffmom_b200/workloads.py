"""Seeded synthetic workloads with the shapes of the benchmark configurations
(no external data): the uneven batch of impedance-loaded surfaces."""
from __future__ import annotations

import math

import numpy as np

from .api import BatchSurface, make_plane_wave
from .mesh import make_circular_plate, make_rect_plate
from .rwg import build_rwg

C0 = 299792458.0


def impedance_surface_batch(count: int = 64, seed: int = 20260004, freq_hz: float = 3e9,
                            n_range=(500, 6000), size_range=(0.5, 3.0)) -> list:
    """`count` rectangular or circular plates, side / diameter ~ U[size_range]
    wavelengths, meshed to the RWG count nearest a target ~ U[n_range]
    (square plates: 3 n^2 - 2 n RWG for n x n cells; disks with Nphi = 4 Nr:
    12 Nr^2 - 8 Nr), per-triangle surface impedance Re ~ U[0, 200] ohm,
    Im ~ U[-300, 300] ohm, one plane wave each (theta ~ U[0, 80) deg,
    phi ~ U[0, 360) deg, theta- or phi-polarised at random)."""
    rng = np.random.default_rng(seed)
    lam = C0 / freq_hz
    k = 2 * math.pi * freq_hz / C0
    out = []
    for _ in range(count):
        disk = bool(rng.integers(2))
        size = rng.uniform(*size_range) * lam
        target = int(rng.integers(n_range[0], n_range[1] + 1))
        if disk:
            nr = max(1, int(round((8 + math.sqrt(64 + 48 * target)) / 24)))
            mesh = make_circular_plate(size / 2, nr, 4 * nr)
        else:
            n = max(1, int(round((2 + math.sqrt(4 + 12 * target)) / 6)))
            mesh = make_rect_plate(size, size, n, n)
        rwg = build_rwg(mesh)
        zs = rng.uniform(0, 200, mesh.ntriangles) + 1j * rng.uniform(-300, 300, mesh.ntriangles)
        th = math.radians(rng.uniform(0, 80))
        ph = math.radians(rng.uniform(0, 360))
        rhat = np.array([math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)])
        if rng.integers(2):
            pol = np.array([math.cos(th) * math.cos(ph), math.cos(th) * math.sin(ph), -math.sin(th)])
        else:
            pol = np.array([-math.sin(ph), math.cos(ph), 0.0])
        out.append(BatchSurface(mesh, rwg, make_plane_wave(-k * rhat, 1.0, pol), zs))
    return out
