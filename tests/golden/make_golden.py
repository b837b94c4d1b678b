"""Writes the golden fixtures of the GPU parity tests from the oracle (the CPU
restatement of the reference algorithm, pinned by tests/test_oracle_golden.py).

    python tests/golden/make_golden.py          # every fixture
    python tests/golden/make_golden.py aca      # aca_plan_plate.npz only

c1_plate.npz -- README minimal case: 0.1 x 0.1 m plate, 6 x 6 cells (72
    triangles, 96 RWG), k = 2 pi / 0.1, quad_order 3: the full Z, the x-pol
    -z plane-wave RHS, the dense-solve currents, the bistatic RCS on the phi = 0
    cut (theta = 0..180 deg step 10) and the monostatic RCS of six seeded
    incidences with their currents.
c2_sphere_sample.npz -- PEC sphere r = 0.5 lambda at 3 GHz, icosphere 5,120
    triangles / 7,680 RWG: 512 seeded Z entries (quad_order 3) and the RHS.
aca_plan_plate.npz -- the H-matrix block plan of a 1 x 1 m plate, 12 x 12
    cells (RWG centres), leaf sizes 4 and 16 at eta 1.5: tree permutation,
    node ranges / children / levels / boxes and the task list, from the
    oracle's restatement of ClusterTree.jl and ACA.jl:696-738.
"""
import math
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "diffmom.jl_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

import oracle as orc  # noqa: E402
from diffmom_b200 import build_rwg, make_icosphere, make_rect_plate  # noqa: E402

C0 = 299792458.0


def waves(k, R, seed):
    rng = np.random.default_rng(seed)
    th = np.deg2rad(rng.uniform(0, 80, R))
    ph = np.deg2rad(rng.uniform(0, 360, R))
    rhat = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], 1)
    tha = np.stack([np.cos(th) * np.cos(ph), np.cos(th) * np.sin(ph), -np.sin(th)], 1)
    pha = np.stack([-np.sin(ph), np.cos(ph), np.zeros(R)], 1)
    pol = np.where((np.arange(R) % 2 == 0)[:, None], tha, pha)
    return -k * rhat, pol


def c1_plate(out):
    mesh = make_rect_plate(0.1, 0.1, 6, 6)
    rwg = build_rwg(mesh)
    k = 2 * math.pi / 0.1
    oc = orc.OracleCache(mesh, rwg, 3)
    Z = oc.assemble_z(k)
    v = oc.plane_wave_rhs([0.0, 0.0, -k], 1.0, [1.0, 0.0, 0.0])
    I = np.linalg.solve(Z, v)
    th = np.deg2rad(np.arange(0, 181, 10.0))
    rhat = np.stack([np.sin(th), np.zeros_like(th), np.cos(th)], 1)
    E = (oc.radiation_vectors(rhat, k) @ I).reshape(-1, 3).T
    sig_cut = 4 * math.pi * np.sum(np.abs(E) ** 2, axis=0)
    kv, pol = waves(k, 6, 3)
    Im, sig_mono = [], []
    for i in range(6):
        Ii = np.linalg.solve(Z, oc.plane_wave_rhs(kv[i], 1.0, pol[i]))
        Ei = oc.radiation_vectors(-kv[i] / k, k) @ Ii
        Im.append(Ii)
        sig_mono.append(4 * math.pi * np.sum(np.abs(Ei) ** 2))
    np.savez_compressed(out, k=k, Z=Z, v=v, I=I, theta=th, sigma_cut=sig_cut, kvecs=kv, pols=pol,
                        I_mono=np.stack(Im, 1), sigma_mono=np.array(sig_mono))


def c2_sample(out):
    lam = C0 / 3e9
    mesh = make_icosphere(0.5 * lam, 4)
    rwg = build_rwg(mesh)
    k = 2 * math.pi / lam
    oc = orc.OracleCache(mesh, rwg, 3)
    rng = np.random.default_rng(7680)
    N = rwg.nedges
    m = rng.integers(1, N + 1, 512)
    n = rng.integers(1, N + 1, 512)
    n[:64] = m[:64]  # self terms
    z = oc.entries(k, m, n)
    v = oc.plane_wave_rhs([0.0, 0.0, -k], 1.0, [1.0, 0.0, 0.0])
    np.savez_compressed(out, k=k, m=m, n=n, z=z, v=v)


def aca_plan(out):
    import aca_oracle as ao
    from diffmom_b200 import rwg_centers
    m = make_rect_plate(1.0, 1.0, 12, 12)
    c = rwg_centers(m, build_rwg(m))
    arrays = {"centers": c}
    for leaf in (4, 16):
        tree = ao.build_cluster_tree(c, leaf)
        tasks = ao.enum_block_tasks(tree, 1.5)
        arrays[f"perm_{leaf}"] = np.asarray(tree.perm, dtype=np.int64)
        arrays[f"nodes_{leaf}"] = np.array([[n.lo, n.hi, n.left, n.right, n.level] for n in tree.nodes], np.int64)
        arrays[f"boxes_{leaf}"] = np.array([list(n.bmin) + list(n.bmax) for n in tree.nodes])
        arrays[f"tasks_{leaf}"] = np.array(tasks, dtype=np.int64)
    np.savez_compressed(out, **arrays)


if __name__ == "__main__":
    here = Path(__file__).resolve().parent
    if len(sys.argv) > 1 and sys.argv[1] == "aca":
        aca_plan(here / "aca_plan_plate.npz")
    else:
        c1_plate(here / "c1_plate.npz")
        c2_sample(here / "c2_sphere_sample.npz")
        aca_plan(here / "aca_plan_plate.npz")
    print("wrote", sorted(p.name for p in here.glob("*.npz")))
