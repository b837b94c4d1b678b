"""The bounded-wait error path, exercised without any GPU fault: the chained
triangular sweeps of a complex128 near-field factor wait on flags published by
earlier CTAs; with DMB_OPT_SPIN_LIMIT = 0 a waiting CTA gives up at its first
poll, records the error bit and returns.  The call must fail with
DMB_ERR_TIMEOUT (DeviceWaitTimeout), and the next call on the same context,
with the default limit, must give the right answer."""
import math

import numpy as np
import pytest

import oracle as orc
from diffmom_b200 import DeviceWaitTimeout, EFIEDevice, build_rwg, make_rect_plate, rwg_centers

pytestmark = pytest.mark.gpu


def test_chain_wait_expires_and_context_recovers():
    m = make_rect_plate(0.1, 0.1, 24, 24)   # 1,680 RWG: 27 chained 64-row blocks
    r = build_rwg(m)
    k = 2 * math.pi / 0.1
    dev = EFIEDevice(m, r)
    dev.assemble(k, precision="fp64")
    cutoff = 0.3 * 0.1
    dev.build_nearfield(cutoff, "lu")
    x = np.random.default_rng(3).standard_normal(r.nedges) * (1 + 0.25j)
    dev.set_option("spin_limit", 0)
    with pytest.raises(DeviceWaitTimeout):
        dev.nf_apply(x)
    dev.set_option("spin_limit", -1)
    y = dev.nf_apply(x)
    c = orc.OracleCache(m, r, 3)
    Znf = orc.nearfield_matrix(c.assemble_z(k), rwg_centers(m, r), cutoff)
    ref = np.linalg.solve(Znf, x)
    err = np.linalg.norm(y - ref) / np.linalg.norm(ref)
    print(f"after the expired wait: near-field apply vs oracle {err:.2e}")
    assert err < 1e-10
    # and a solve on the same context still converges
    v = c.plane_wave_rhs([0, 0, -k], 1.0, [1, 0, 0])
    I, st = dev.gmres(v, tol=1e-8, maxiter=200, preconditioner=dev.preconditioner)
    assert st.solved and st.true_residual <= 1e-8
    dev.close()
