"""Learned near-field right preconditioner: gradient check of the hand-written
training kernels against a torch-CPU autograd restatement of the same network,
checkpoint round trip, and the ablation that shows what the trained network
gains over the plain local-inverse rows (with the near-field LDL^T and no
preconditioner beside it).  The FP64 true residual is the criterion."""
import math

import numpy as np
import pytest

from diffmom_b200 import EFIEDevice, build_rwg, make_perturbed_ellipsoid, make_rect_plate

pytestmark = pytest.mark.gpu

C0 = 299792458.0
NF, NH, KS = 13, 32, 64


def _unpack(P):
    import torch
    o = 0
    W1 = P[o:o + NH * NF].reshape(NH, NF); o += NH * NF
    b1 = P[o:o + NH]; o += NH
    W2 = P[o:o + NH * 2 * NH].reshape(NH, 2 * NH); o += NH * 2 * NH
    b2 = P[o:o + NH]; o += NH
    W3 = P[o:o + 2 * NH].reshape(2, NH); o += 2 * NH
    b3 = P[o:o + 2]; o += 2
    assert o == P.numel()
    return W1, b1, W2, b2, W3, b3


def _torch_loss(P, feat, tgt, wgt, cnt):
    import torch
    W1, b1, W2, b2, W3, b3 = _unpack(P)
    total = 0
    for b in range(feat.shape[0]):
        k = int(cnt[b])
        f = feat[b, :k]
        h = torch.tanh(f @ W1.T + b1)
        ctx = h.mean(0, keepdim=True).expand(k, NH)
        g = torch.tanh(torch.cat([h, ctx], 1) @ W2.T + b2)
        out = g @ W3.T + b3
        total = total + (wgt[b, :k, None] * (out - tgt[b, :k]) ** 2).sum()
    return total / feat.shape[0]


def test_network_gradient_matches_torch_cpu():
    import torch
    m = make_rect_plate(0.1, 0.1, 2, 2)
    dev = EFIEDevice(m, build_rwg(m))
    npar = dev.ctx.lib.dmb_net_param_count()
    rng = np.random.default_rng(0)
    P = (rng.standard_normal(npar) * 0.3).astype(np.float32)
    dev.set_network_weights(P)
    nrows = 6
    cnt = np.array([64, 1, 17, 40, 64, 5], dtype=np.int32)
    feat = rng.standard_normal((nrows, KS, NF)).astype(np.float32)
    tgt = (rng.standard_normal((nrows, KS, 2)) * 0.1).astype(np.float32)
    for b in range(nrows):
        feat[b, cnt[b]:] = 0
        tgt[b, cnt[b]:] = 0
    wgt = rng.uniform(0.5, 2.0, (nrows, KS)).astype(np.float32)
    grad = np.empty(npar, dtype=np.float32)
    loss = np.empty(1, dtype=np.float32)
    from diffmom_b200 import _native as nat
    dev.ctx.call("dmb_net_loss_grad", feat.ctypes.data_as(nat._FP), tgt.ctypes.data_as(nat._FP),
                 wgt.ctypes.data_as(nat._FP), cnt.ctypes.data_as(nat._IP), nrows,
                 grad.ctypes.data_as(nat._FP), loss.ctypes.data_as(nat._FP))
    Pt = torch.tensor(P.astype(np.float64), requires_grad=True)
    lt = _torch_loss(Pt, torch.tensor(feat, dtype=torch.float64), torch.tensor(tgt, dtype=torch.float64),
                     torch.tensor(wgt, dtype=torch.float64), cnt)
    lt.backward()
    gref = Pt.grad.numpy()
    assert abs(loss[0] - lt.item()) <= 1e-4 * abs(lt.item())
    assert np.linalg.norm(grad - gref) <= 1e-4 * np.linalg.norm(gref)
    # per block of parameters too (tiny blocks like b3 included)
    assert np.allclose(grad, gref, rtol=2e-3, atol=1e-5 * np.abs(gref).max())
    dev.close()


def test_network_checkpoint_round_trip(tmp_path):
    m = make_rect_plate(0.1, 0.1, 2, 2)
    dev = EFIEDevice(m, build_rwg(m))
    w = dev.network_weights()
    w2 = (w + 0.5).astype(np.float32)
    dev.set_network_weights(w2)
    p = tmp_path / "net.bin"
    dev.save_network(p)
    dev.set_network_weights(w)
    dev.load_network(p)
    assert np.array_equal(dev.network_weights(), w2)
    with pytest.raises(ValueError):
        (tmp_path / "bad.bin").write_bytes(b"garbage!" + b"\0" * 8)
        dev.load_network(tmp_path / "bad.bin")
    dev.close()


def _iters(dev, v, P, side="right", maxiter=600):
    x, st = dev.gmres(v, tol=1e-6, maxiter=maxiter, preconditioner=P, precond_side=side)
    assert st.solved and st.true_residual <= 2e-6, st
    return st.niter, x.reshape(-1)


def test_learned_preconditioner_ablation():
    """What the trained network gains over the same method without it, on a
    body none of the training bodies is: the library's default weights
    (trained on the GPU over 48 generated perturbed ellipsoids, seeds
    1000-1047) against the plain ring step (the learned step with the network
    switched off), the exact local inverse, the near-field LDL^T and no
    preconditioner; GMRES to 1e-6 checked on the FP64 residual."""
    from diffmom_b200.learned import DEFAULT_WEIGHTS
    lam = C0 / 3e9
    k = 2 * math.pi / lam
    r = 0.2 * lam
    test_body = make_perturbed_ellipsoid(lam, 99, frequency=8)   # 1,920 RWG
    trwg = build_rwg(test_body)
    dev = EFIEDevice(test_body, trwg)
    dev.load_network(DEFAULT_WEIGHTS)
    dev.assemble(k, precision="mixed")
    v = dev.plane_wave_rhs([[0, 0, -k]], [1.0], [[1, 0, 0]])[:, 0]
    it_none, x_none = _iters(dev, v, None)
    it_local, x_local = _iters(dev, v, dev.build_local(r, learned=False))
    it_ring, x_ring = _iters(dev, v, dev.build_local(r, mode="ring"))
    it_learned, x_learned = _iters(dev, v, dev.build_local(r, learned=True))
    it_ls, x_ls = _iters(dev, v, dev.build_local(r, mode="ls"))
    it_nf, x_nf = _iters(dev, v, dev.build_nearfield(0.2 * lam, "lu"), side="left")
    print(f"GMRES iterations: none {it_none}, near-field LDL^T {it_nf}, local inverse {it_local}, "
          f"ring step {it_ring}, learned ring step {it_learned}, least-squares target {it_ls}")
    for x in (x_local, x_learned, x_nf):
        assert np.linalg.norm(x - x_none) / np.linalg.norm(x_none) < 1e-4
    assert it_local < it_none
    assert it_ring < it_local
    # the network's gain: strictly fewer iterations than the plain ring step,
    # and at least 10 % fewer than the exact local inverse
    assert it_learned < it_ring
    assert it_learned <= 0.9 * it_local
    dev.close()


def test_training_streams_generated_bodies():
    """GPU training over a stream of generated bodies (forward, backward and
    Adam on the device) from the untrained network: finite losses, weights
    that change, and a learned preconditioner that converges with them."""
    from diffmom_b200.learned import train_learned_network, training_bodies
    m = make_rect_plate(0.1, 0.1, 2, 2)
    dev = EFIEDevice(m, build_rwg(m))
    w0 = dev.network_weights()
    rep = train_learned_network(dev, training_bodies(6, frequencies=(6, 7)), epochs=2)
    assert rep.bodies == 6 and rep.rwg_total > 0
    assert all(np.isfinite(rep.losses))
    assert not np.array_equal(dev.network_weights(), w0)
    lam = C0 / 3e9
    k = 2 * math.pi / lam
    dev.assemble(k, precision="mixed")
    v = dev.plane_wave_rhs([[0, 0, -k]], [1.0], [[1, 0, 0]])[:, 0]
    _iters(dev, v, dev.build_local(0.2 * lam, learned=True))
    dev.close()
