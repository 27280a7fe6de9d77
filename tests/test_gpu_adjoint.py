"""Adjoint of the fixed-assignment reconstruction loss (kilosort_b200.adjoint).

Checks, against the float64 torch reference in oracle/adjoint.py:
* the forward residual and loss;
* gradients w.r.t. U, wPCA and amplitudes against torch.autograd in float64
  (relative error of each gradient <= 1e-4 of its largest entry);
* the configuration-4 check: C=384, K=600, one 60000-sample batch with the
  spikes of the FP32 matcher (~25000), gradients on 50 random coordinates
  against float64 central finite differences with eps = 1e-4, relative error
  <= 1e-3 (the loss is quadratic in each parameter group, so the central
  difference is exact up to rounding);
* determinism and the scaling by the upstream gradient.
"""
import numpy as np
import pytest
import torch

import kilosort_b200 as kb
from kilosort_b200 import synth
from kilosort_b200.adjoint import reconstruct, reconstruction_loss
from oracle import adjoint as oa

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _matched(rec, b=0, Th=8.0):
    U = torch.from_numpy(rec.U).to(DEV)
    W = torch.from_numpy(rec.wPCA).to(DEV)
    X = torch.from_numpy(np.ascontiguousarray(rec.batch(b))).to(DEV)
    ops = dict(Th_learned=Th, nt=rec.nt, max_peels=100, wPCA=W)
    ctc = kb.prepare_matching(ops, U)
    st, amps, _, Xres = kb.run_matching(ops, X, U, ctc, device=DEV)
    return X, U, W, st, amps.reshape(-1), Xres


def _perturbed(U, W, amps, seed=0):
    """A point away from the matcher's fixed point (refinement starts there)."""
    g = torch.Generator(device=DEV).manual_seed(seed)
    amps_p = amps * (1 + 0.1 * torch.randn(amps.shape, generator=g, device=DEV))
    U_p = U + 0.05 * U.abs().mean() * torch.randn(U.shape, generator=g, device=DEV)
    W_p = W + 0.01 * torch.randn(W.shape, generator=g, device=DEV)
    return U_p, W_p, amps_p


def _small():
    rec = synth.make_recording(4101, n_chan=64, n_templates=40, batch_lengths=[6000],
                               rate_hz=(10.0, 30.0))
    return _matched(rec)


def test_forward_matches_reference_and_peel_residual(cuda_device):
    X, U, W, st, amps, Xres_peel = _small()
    assert len(st) > 50
    Xres, loss = reconstruct(X, st, amps, U, W)
    ref = oa.recon_residual(X.double(), st, amps.double(), U.double(), W.double())
    ref_loss = float((ref ** 2).sum())
    assert abs(float(loss) - ref_loss) <= 1e-6 * ref_loss
    assert torch.allclose(Xres.double(), ref, atol=2e-5, rtol=0)
    # the peel subtracts the same waveforms (in record order instead of time
    # order): the same residual up to the order of float32 subtractions
    assert torch.allclose(Xres, Xres_peel, atol=2e-5, rtol=0)
    # and the autograd entry gives the same loss
    assert float(reconstruction_loss(X, st, amps, U, W)) == pytest.approx(float(loss), rel=1e-6)


@pytest.mark.parametrize("perturb", [False, True])
def test_gradients_match_autograd_float64(cuda_device, perturb):
    X, U, W, st, amps, _ = _small()
    if perturb:
        U, W, amps = _perturbed(U, W, amps)
    Uq = U.clone().requires_grad_(True)
    Wq = W.clone().requires_grad_(True)
    aq = amps.clone().requires_grad_(True)
    reconstruction_loss(X, st, aq, Uq, Wq).backward()
    Ud = U.double().requires_grad_(True)
    Wd = W.double().requires_grad_(True)
    ad = amps.double().requires_grad_(True)
    oa.recon_loss(X.double(), st, ad, Ud, Wd).backward()
    for got, ref, name in ((Uq.grad, Ud.grad, "U"), (Wq.grad, Wd.grad, "wPCA"),
                           (aq.grad, ad.grad, "amps")):
        scale = ref.abs().max().item()
        err = (got.double() - ref).abs().max().item()
        assert err <= 1e-4 * scale, (name, err, scale)


def test_deterministic_and_scaled_by_upstream_gradient(cuda_device):
    X, U, W, st, amps, _ = _small()
    U, W, amps = _perturbed(U, W, amps, seed=1)
    grads = []
    for mult in (1.0, 1.0, 3.0):
        Uq = U.clone().requires_grad_(True)
        Wq = W.clone().requires_grad_(True)
        aq = amps.clone().requires_grad_(True)
        (mult * reconstruction_loss(X, st, aq, Uq, Wq)).backward()
        grads.append((Uq.grad, Wq.grad, aq.grad))
    for a, b in zip(grads[0], grads[1]):
        assert torch.equal(a, b)
    for a, c in zip(grads[0], grads[2]):
        assert torch.allclose(3.0 * a, c, rtol=1e-6, atol=1e-6 * a.abs().max().item())


def test_out_of_range_spike_is_rejected(cuda_device):
    X, U, W, st, amps, _ = _small()
    bad = st.clone()
    bad[0, 0] = X.shape[1] + 5
    with pytest.raises(kb._lib.KilosortB200Error):
        reconstruction_loss(X, bad, amps, U, W)


def test_config4_finite_differences(cuda_device):
    rec = synth.config_recording(4)
    X, U, W, st, amps, _ = _matched(rec)
    assert len(st) > 20000, len(st)
    U, W, amps = _perturbed(U, W, amps, seed=4)
    Uq = U.clone().requires_grad_(True)
    Wq = W.clone().requires_grad_(True)
    aq = amps.clone().requires_grad_(True)
    reconstruction_loss(X, st, aq, Uq, Wq).backward()
    Xd, Ud, Wd, ad = X.double(), U.double(), W.double(), amps.double()

    def loss64(Ux, Wx, ax):
        return float(oa.recon_loss(Xd, st, ax, Ux, Wx))

    rng = np.random.default_rng(44)
    eps = 1e-4
    checks = []
    # 50 coordinates: 20 of U (on templates that fire), 15 of wPCA, 15 amplitudes
    fired = torch.unique(st[:, 1]).cpu().numpy()
    for _ in range(20):
        k = int(rng.choice(fired))
        p, c = int(rng.integers(U.shape[1])), int(rng.integers(U.shape[2]))
        e = torch.zeros_like(Ud)
        e[k, p, c] = eps
        fd = (loss64(Ud + e, Wd, ad) - loss64(Ud - e, Wd, ad)) / (2 * eps)
        checks.append(("U", fd, float(Uq.grad[k, p, c])))
    for _ in range(15):
        p, t = int(rng.integers(W.shape[0])), int(rng.integers(W.shape[1]))
        e = torch.zeros_like(Wd)
        e[p, t] = eps
        fd = (loss64(Ud, Wd + e, ad) - loss64(Ud, Wd - e, ad)) / (2 * eps)
        checks.append(("wPCA", fd, float(Wq.grad[p, t])))
    for _ in range(15):
        s = int(rng.integers(len(amps)))
        e = torch.zeros_like(ad)
        e[s] = eps
        fd = (loss64(Ud, Wd, ad + e) - loss64(Ud, Wd, ad - e)) / (2 * eps)
        checks.append(("amps", fd, float(aq.grad[s])))
    # relative error per coordinate; the floor (1e-2 of the group's typical
    # magnitude) keeps coordinates whose gradient is nearly zero meaningful
    for group in ("U", "wPCA", "amps"):
        vals = [(fd, g) for n, fd, g in checks if n == group]
        typical = float(np.median([abs(fd) for fd, _ in vals]))
        for fd, g in vals:
            rel = abs(g - fd) / max(abs(fd), 1e-2 * typical)
            assert rel <= 1e-3, (group, fd, g, rel)
