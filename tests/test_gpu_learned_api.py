"""solve_scattering with the learned right preconditioner (the library's
default weights, trained over generated bodies by diffmom_b200.learned) and
its near-field LU fallback, against the near-field LU path on the same body.
The unpreconditioned FP64 residual is the criterion of every solve."""
import math

import numpy as np
import pytest

from diffmom_b200 import build_rwg, make_perturbed_ellipsoid, make_plane_wave, solve_scattering
from diffmom_b200.learned import DEFAULT_WEIGHTS

pytestmark = pytest.mark.gpu

C0 = 299792458.0
F = 3e9
LAM = C0 / F
K = 2 * math.pi / LAM


def _body(seed=77, frequency=10):
    m = make_perturbed_ellipsoid(LAM, seed, frequency=frequency)
    return m, build_rwg(m)


def test_default_weights_are_shipped():
    assert DEFAULT_WEIGHTS.exists()
    assert DEFAULT_WEIGHTS.stat().st_size == 8 + 4 + 4 * 2594


def test_solve_scattering_learned_matches_nearfield_lu():
    m, r = _body()
    exc = make_plane_wave([0.0, 0.0, -K], 1.0, [1.0, 0.0, 0.0])
    kw = dict(method="dense_gmres", precision="mixed", gmres_tol=1e-6, rwg=r)
    ref = solve_scattering(m, F, exc, preconditioner="lu", nf_cutoff_lambda=0.2, **kw)
    loc = solve_scattering(m, F, exc, preconditioner="local", **kw)
    lrn = solve_scattering(m, F, exc, preconditioner="learned", **kw)
    for res in (ref, loc, lrn):
        assert res.true_residual <= 1e-6, res
    assert not lrn.warnings or all("did not converge" not in w for w in lrn.warnings)
    d = np.linalg.norm(lrn.I_coeffs - ref.I_coeffs) / np.linalg.norm(ref.I_coeffs)
    assert d < 1e-4, d
    print(f"N={r.nedges}: GMRES iterations near-field LU (left) {ref.gmres_iters}, local {loc.gmres_iters}, "
          f"learned {lrn.gmres_iters}")
    assert lrn.gmres_iters < loc.gmres_iters


def test_learned_falls_back_to_nearfield_lu():
    m, r = _body(seed=78, frequency=8)
    exc = make_plane_wave([0.0, 0.0, -K], 1.0, [1.0, 0.0, 0.0])
    res = solve_scattering(m, F, exc, method="dense_gmres", precision="mixed", preconditioner="learned",
                           gmres_tol=1e-6, gmres_maxiter=3, nf_cutoff_lambda=math.inf, rwg=r)
    assert any("fell back" in w or "near-field LU" in w for w in res.warnings), res.warnings
    assert res.true_residual <= 1e-6


def test_learned_rejects_the_aca_path():
    m, r = _body(seed=79, frequency=6)
    exc = make_plane_wave([0.0, 0.0, -K], 1.0, [1.0, 0.0, 0.0])
    with pytest.raises(ValueError):
        solve_scattering(m, F, exc, method="aca_gmres", preconditioner="learned", rwg=r)
