"""Streaming front end: int16 whitening on the tensor cores, batch cutting as
kilosort/io.py does it, and the streamed matcher against one run_matching per
whitened batch (same kernels on the same whitened input: identical spikes)."""
import numpy as np
import pytest
import torch

import kilosort_b200 as kb
from kilosort_b200 import synth
from kilosort_b200.stream import StreamMatcher, Whitener, batch_windows, padded_raw_window

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _mixing(C, seed=0):
    """A banded, well-conditioned channel mixing M; whitening is M^-1."""
    rng = np.random.default_rng(seed)
    M = np.eye(C)
    for d in (1, 2):
        v = 0.25 / d * (1 + 0.2 * rng.standard_normal(C - d))
        M += np.diag(v, d) + np.diag(v, -d)
    return M


def test_whitening_matches_float64(cuda_device):
    rng = np.random.default_rng(5)
    T, C = 5000, 64
    raw = rng.integers(-30000, 30000, size=(T, C), dtype=np.int16)
    Wrot = torch.from_numpy(rng.standard_normal((C, C)) / np.sqrt(C)).float()
    scale = 1e-3
    w = Whitener(Wrot, scale, T, DEV)
    X = torch.empty((C, T), device=DEV)
    w(torch.from_numpy(raw).to(DEV), X)
    ref = (scale * Wrot.double()) @ torch.from_numpy(raw).double().T
    err = (X.double().cpu() - ref).abs().max().item() / ref.abs().max().item()
    assert err < 3e-5, err
    assert w.status()[0] == 0


def _raw_recording(seed=6001, C=64, K=40, NT=3000, nb=5):
    rec = synth.make_recording(seed, n_chan=C, probe="np1", n_templates=K,
                               batch_lengths=[NT] * nb, rate_hz=(10.0, 30.0))
    M = _mixing(C, seed)
    raw = np.round(200.0 * (M @ rec.signal.astype(np.float64))).T
    raw = np.clip(raw, -32768, 32767).astype(np.int16)
    Wrot = torch.from_numpy(np.linalg.inv(M)).float()
    return rec, raw, Wrot, 1.0 / 200.0


def test_stream_equals_per_batch_matching(cuda_device):
    NT = 3000
    rec, raw, Wrot, scale = _raw_recording(NT=NT)
    U = torch.from_numpy(rec.U).to(DEV)
    W = torch.from_numpy(rec.wPCA).to(DEV)
    ops = dict(Th_learned=8.0, nt=rec.nt, max_peels=100, wPCA=W)
    sm = StreamMatcher(raw, Wrot, scale, ops, U, NT=NT, group=2, teams=2)
    times, templ, amps, bidx = sm.run()
    sm.close()
    assert len(times) > 100
    # one run_matching per whitened batch
    w = Whitener(Wrot, scale, NT + 2 * rec.nt, DEV)
    ctc = kb.prepare_matching(ops, U)
    nt = rec.nt
    ref_t, ref_k = [], []
    for b in range(len(batch_windows(raw.shape[0], NT, nt))):
        win = padded_raw_window(raw, b, NT, nt, np.empty((NT + 2 * nt, raw.shape[1]), np.int16))
        X = torch.empty((raw.shape[1], NT + 2 * nt), device=DEV)
        w(torch.from_numpy(win).to(DEV), X)
        st, _, _, _ = kb.run_matching(dict(ops, projection="bf16x3"), X, U, ctc, device=DEV)
        st = st.cpu().numpy()
        ref_t.append(st[:, 0] - nt + b * NT)
        ref_k.append(st[:, 1])
    np.testing.assert_array_equal(times, np.concatenate(ref_t))
    np.testing.assert_array_equal(templ, np.concatenate(ref_k))
    # the whitened stream recovers the synthetic units: a found spike of the
    # same unit within 3 samples of most true troughs (trough = tau - nt//2 + 20)
    trough = times - nt // 2 + 20
    hits = 0
    for t, k in zip(rec.spike_times.tolist(), rec.spike_units.tolist()):
        sel = np.abs(trough - t) <= 3
        hits += bool(np.any(templ[sel] == k))
    assert hits >= 0.5 * len(rec.spike_times), (hits, len(rec.spike_times))


def test_stream_refinement_updates_templates(cuda_device):
    rec, raw, Wrot, scale = _raw_recording(seed=6002)
    U = torch.from_numpy(rec.U).to(DEV)
    U0 = U.clone()
    W = torch.from_numpy(rec.wPCA).to(DEV)
    ops = dict(Th_learned=8.0, nt=rec.nt, max_peels=100, wPCA=W)
    sm = StreamMatcher(raw, Wrot, scale, ops, U, NT=3000, group=2, teams=2, refine_every=1,
                       refine_lr=1e-6)
    times, templ, amps, bidx = sm.run()
    sm.close()
    assert sm.refinements >= 2
    assert not torch.equal(U, U0)
    # only each template's footprint moves (channels within 1e-3 of its peak norm)
    norm = U0.norm(dim=1)
    off = (norm < 1e-3 * norm.amax(dim=1, keepdim=True)).unsqueeze(1).expand_as(U)
    assert off.any() and torch.equal(U[off], U0[off])
    assert len(times) > 100
    # ctc follows the refined templates
    ctc_now = kb.prepare_matching(ops, U)
    assert torch.allclose(ctc_now, sm.ctc, rtol=0, atol=1e-5 * ctc_now.abs().max().item())
