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
