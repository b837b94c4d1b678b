"""dmb_matvec_free_noalloc: the matrix-free product for callers that cannot
allocate device memory mid-run (their device memory belongs to an external
pool, or their budget forbids allocation after set-up).  It must give the same
product as the allocating entry point dmb_matvec_free, call after call, while
the caller owns the input and output device buffers.

This file sorts last so that a run stopping at the first failure has already
run every other test."""
import ctypes
import math

import numpy as np
import pytest

from diffmom_b200 import build_rwg, make_icosphere, make_rect_plate, matrixfree_efie_operator
from diffmom_b200 import _native as nat

pytestmark = pytest.mark.gpu

TOL = 1e-12  # same kernels; only the order of the near-term additions may differ


def _noalloc(op, x):
    import torch
    xd = torch.from_numpy(np.ascontiguousarray(x).view(np.float64)).to("cuda:0")
    yd = torch.full_like(xd, float("nan"))
    torch.cuda.synchronize()
    st = op.dev.ctx.lib.dmb_matvec_free_noalloc(op.dev.ctx.h, ctypes.c_void_p(xd.data_ptr()),
                                                 ctypes.c_void_p(yd.data_ptr()))
    op.dev.ctx._check(st)
    torch.cuda.synchronize()
    return yd.cpu().numpy().view(np.complex128)


def test_noalloc_matches_allocating_entry_point_two_calls():
    m = make_icosphere(0.05, 2)
    r = build_rwg(m)
    k = 2 * math.pi * 2e9 / 299792458.0
    op = matrixfree_efie_operator(m, r, k)
    rng = np.random.default_rng(11)
    for _ in range(2):  # two calls in a row share (and reuse) the static scratch
        x = rng.standard_normal(r.nedges) + 1j * rng.standard_normal(r.nedges)
        y_ref = op @ x
        y = _noalloc(op, x)
        assert np.all(np.isfinite(y))
        assert np.linalg.norm(y - y_ref) / np.linalg.norm(y_ref) < TOL


def test_noalloc_at_the_maximum_mesh_size():
    # exactly 32,768 triangles (128 x 128 plate): the output half starts at
    # slot 3 x 32,768 and the last slots of both halves are used
    m = make_rect_plate(1.0, 1.0, 128, 128)
    assert m.ntriangles == 32768
    r = build_rwg(m)
    op = matrixfree_efie_operator(m, r, 2 * math.pi)
    rng = np.random.default_rng(12)
    for _ in range(2):
        x = rng.standard_normal(r.nedges) + 1j * rng.standard_normal(r.nedges)
        y_ref = op @ x
        y = _noalloc(op, x)
        assert np.all(np.isfinite(y))
        assert np.linalg.norm(y - y_ref) / np.linalg.norm(y_ref) < TOL


def test_noalloc_rejects_meshes_above_the_maximum():
    m = make_rect_plate(1.0, 1.0, 130, 130)  # 33,800 triangles > 32,768
    r = build_rwg(m)
    op = matrixfree_efie_operator(m, r, 2 * math.pi)
    x = np.ones(r.nedges, dtype=np.complex128)
    with pytest.raises(ValueError, match="at most 32768 triangles"):
        _noalloc(op, x)
