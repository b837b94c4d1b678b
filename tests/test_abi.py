"""CPU checks of the C ABI boundary: the library loads, exports every symbol the
header declares, and refuses to create a context without a GPU (no silent CPU
fallback)."""
import ctypes

import pytest

from conftest import has_gpu
from diffmom_b200 import _native as nat


def test_library_exports_every_declared_symbol():
    lib = nat.load_library()
    declared = nat.declared_symbols()
    assert len(declared) >= 19
    for name in declared:
        assert hasattr(lib, name), name
    assert lib.dmb_version().startswith(b"diffmom_b200")


def test_signatures_cover_header():
    assert set(nat.declared_symbols()) <= set(nat.SIGNATURES)


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU failure mode")
def test_context_creation_fails_loudly_without_gpu():
    lib = nat.load_library()
    h = ctypes.c_void_p()
    assert lib.dmb_ctx_create(0, ctypes.byref(h)) == nat.DMB_ERR_CUDA
    with pytest.raises(nat.DiffMoMError):
        nat.Context(0)


def test_missing_library_raises(tmp_path):
    with pytest.raises(nat.DiffMoMError):
        nat.load_library(tmp_path / "absent.so")


def test_solve_scattering_method_selection_and_payload_guard_on_cpu():
    # Workflow.jl:108-119 argument checks and :169-174 payload limit, all
    # raised before any device work
    import math
    from diffmom_b200 import make_plane_wave, make_rect_plate, solve_scattering
    m = make_rect_plate(0.1, 0.1, 6, 6)   # 96 RWG
    f = 299792458.0 / 0.1
    pw = make_plane_wave([0, 0, -2 * math.pi / 0.1], 1.0, [1, 0, 0])
    with pytest.raises(ValueError, match="max_dense_matrix_bytes"):
        solve_scattering(m, f, pw, method="dense_gmres", max_dense_matrix_bytes=96 * 96 * 16 - 1)
    with pytest.raises(ValueError, match="max_dense_matrix_bytes"):
        solve_scattering(m, f, pw, method="dense_direct", precision="mixed", max_dense_matrix_bytes=96 * 96 * 8 - 1)
    with pytest.raises(ValueError, match="mlfma_threshold"):
        solve_scattering(m, f, pw, dense_direct_limit=0, dense_gmres_limit=0, mlfma_threshold=10)
    with pytest.raises(ValueError, match="dense_gmres_limit"):
        solve_scattering(m, f, pw, dense_direct_limit=100, dense_gmres_limit=50)
    with pytest.raises(ValueError, match="mlfma"):
        solve_scattering(m, f, pw, method="mlfma")
    with pytest.raises(ValueError, match="surface_impedance"):
        solve_scattering(m, f, pw, dense_direct_limit=0, dense_gmres_limit=50, surface_impedance=1.0)
