"""GMRES iterations replayed as captured CUDA graphs (DMB_OPT_GMRES_GRAPHS):
repeated solves -- direct launches on the first meeting of an iteration
range, capture on the second, replay afterwards -- give bitwise the same
iterates as direct launches, for several preconditioners and both sides."""
import math

import numpy as np
import pytest

import oracle as orc
from diffmom_b200 import EFIEDevice, build_rwg, make_rect_plate

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def plate():
    m = make_rect_plate(0.2, 0.2, 14, 14)
    rwg = build_rwg(m)
    k = 2 * math.pi / 0.1
    v = orc.OracleCache(m, rwg, 3).plane_wave_rhs([0, 0, -k], 1.0, [1, 0, 0])
    return m, rwg, k, v


@pytest.mark.parametrize("pc,side", [(None, "left"), ("diag", "left"), ("lu", "right"), ("local", "right")])
def test_graph_replay_matches_direct_launches(plate, pc, side):
    m, rwg, k, v = plate
    runs = {}
    for graphs in (0, 1):
        dev = EFIEDevice(m, rwg)
        dev.set_option("gmres_graphs", graphs)
        dev.assemble(k, precision="mixed")
        P = None
        if pc == "local":
            P = dev.build_local(0.1, mode="local")
        elif pc is not None:
            P = dev.build_nearfield(0.05, pc)
        out = []
        for _ in range(4):  # direct, capture, replay, replay
            x, st = dev.gmres(v, tol=1e-8, maxiter=200, preconditioner=P, precond_side=side)
            out.append((x.copy(), st.niter))
        dev.close()
        runs[graphs] = out
    x0, n0 = runs[0][0]
    for graphs in (0, 1):
        for x, n in runs[graphs]:
            assert n == n0
            np.testing.assert_array_equal(x, x0)
