"""Device preprocessing (ks_preprocess_int16) against the reference's filter.

* the golden cases (the reference's own BinaryFiltered.filter outputs,
  tests/golden/golden_pre.npz): max |X - X_ref| <= 1e-4 of max |X_ref| (the
  whitening runs in split-BF16, ~2^-16 per product; the FP32 circular FIR
  and the exact mean stay near 1e-7); the artifact case is all zeros with the
  artifact flag set;
* a full-size batch (385 file channels, 384 mapped, L = 60122, CAR, high-pass,
  whitening with a drift matrix) against the oracle in float64, same bound;
* a channel map entry outside the file's channels is reported (KS_ERR_ARG in
  the status word), nothing is read out of bounds;
* the stream with preprocessing equals one run_matching per preprocessed
  padded batch.
"""
import hashlib

import numpy as np
import pytest
import torch

import kilosort_b200 as kb
from kilosort_b200 import _lib, synth
from kilosort_b200.preprocess import Preprocessor
from kilosort_b200.stream import StreamMatcher, batch_windows, padded_raw_window
from oracle import preprocess as op
from tests.golden import make_golden_pre as mk

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
G = np.load(mk.__file__.replace("make_golden_pre.py", "golden_pre.npz"))


@pytest.mark.parametrize("name", list(mk.CASES))
def test_golden_cases(cuda_device, name):
    seed, L, inv, car, use_hp, use_w, shift = G[f"{name}_params"]
    raw = synth.raw_batch(int(seed), int(G["n_chan_bin"]), int(L))
    assert hashlib.sha256(raw.tobytes()).hexdigest()[:16] == str(G[f"{name}_raw_sha"])
    drift = None
    if shift >= 0:
        drift = op.drift_matrix(G[f"{name}_xc"], G[f"{name}_yc"], float(shift)).float()
    p = Preprocessor(int(G["n_chan_bin"]), int(L),
                     whiten=torch.from_numpy(G[f"{name}_W"]) if use_w else None,
                     chan_map=G["chan_map"], hp_filter=op.highpass_filter() if use_hp else None,
                     do_CAR=bool(car), invert_sign=bool(inv),
                     artifact_threshold=float(G[f"{name}_thr"]), device=DEV)
    X = p(torch.from_numpy(raw).to(DEV), drift=drift).cpu().numpy()
    status, artifact = p.status()
    assert status == _lib.KS_OK
    ref = G[f"{name}_out"]
    if name == "artifact":
        assert artifact and not X.any()
        return
    assert not artifact
    err = np.abs(X - ref).max()
    assert err <= 1e-4 * np.abs(ref).max(), (name, err, np.abs(ref).max())


def test_full_size_with_drift(cuda_device):
    n_bin, L = 385, 60122
    raw = synth.raw_batch(7101, n_bin, L, n_spikes=3000)
    cmap = np.delete(np.arange(n_bin), 200)
    C = len(cmap)
    rng = np.random.default_rng(3)
    W = (np.eye(C) + 0.05 * rng.standard_normal((C, C))).astype(np.float32)
    xc = np.tile(np.array([43.0, 11.0, 59.0, 27.0]), C // 4)
    yc = 20.0 * (np.arange(C) // 2)
    M = op.drift_matrix(xc, yc, 4.0)
    hp = op.highpass_filter()
    p = Preprocessor(n_bin, L, whiten=torch.from_numpy(W), chan_map=cmap, hp_filter=hp,
                     device=DEV)
    X = p(torch.from_numpy(raw).to(DEV), drift=M.float()).cpu().numpy()
    assert p.status() == (_lib.KS_OK, False)
    ref = op.filter_batch(torch.from_numpy(raw.T.astype(np.float64)),
                          chan_map=torch.from_numpy(cmap), hp=hp.double(),
                          whiten=torch.from_numpy(W).double(), drift=M.double()).numpy()
    err = np.abs(X - ref).max()
    assert err <= 1e-4 * np.abs(ref).max(), (err, np.abs(ref).max())


def test_bad_channel_map_is_reported(cuda_device):
    raw = synth.raw_batch(7102, 16, 1100)
    p = Preprocessor(16, 1100, chan_map=np.array([0, 1, 2, 16]), device=DEV)
    p(torch.from_numpy(raw).to(DEV))
    assert p.status()[0] == _lib.KS_ERR_ARG


def test_stream_with_preprocessing_equals_per_batch(cuda_device):
    NT = 3000
    rec = synth.make_recording(6101, n_chan=64, probe="np1", n_templates=40,
                               batch_lengths=[NT] * 4, rate_hz=(10.0, 30.0))
    n_bin = 66
    cmap = np.arange(1, 65)                      # file channels 1..64
    noise = synth.raw_batch(6102, n_bin, rec.signal.shape[1])
    raw = noise.astype(np.float64)
    raw[:, cmap] += np.round(25.0 * rec.signal.T)
    raw = np.clip(raw, -32768, 32767).astype(np.int16)
    U = torch.from_numpy(rec.U).to(DEV)
    W = torch.from_numpy(rec.wPCA).to(DEV)
    ops = dict(Th_learned=8.0, nt=rec.nt, max_peels=100, wPCA=W)
    Wrot = torch.eye(64) / 25.0
    pre = dict(chan_map=cmap, hp_filter=op.highpass_filter(), do_CAR=True)
    sm = StreamMatcher(raw, Wrot, 1.0, ops, U, NT=NT, group=2, teams=2, preprocess=pre)
    times, templ, amps, bidx = sm.run()
    sm.close()
    assert len(times) > 50
    nt = rec.nt
    L = NT + 2 * nt
    p = Preprocessor(n_bin, L, whiten=Wrot, device=DEV, **pre)
    ctc = kb.prepare_matching(ops, U)
    ref_t, ref_k = [], []
    for b in range(len(batch_windows(raw.shape[0], NT, nt))):
        win = padded_raw_window(raw, b, NT, nt, np.empty((L, n_bin), np.int16))
        X = p(torch.from_numpy(win).to(DEV))
        st, _, _, _ = kb.run_matching(dict(ops, projection="bf16x3"), X, U, ctc, device=DEV)
        st = st.cpu().numpy()
        ref_t.append(st[:, 0] - nt + b * NT)
        ref_k.append(st[:, 1])
    np.testing.assert_array_equal(times, np.concatenate(ref_t))
    np.testing.assert_array_equal(templ, np.concatenate(ref_k))


def test_single_channel_and_odd_length(cuda_device):
    """C = 1 (no CAR: the median of one channel is itself), odd batch length
    with the high-pass, against the oracle in float64."""
    raw = synth.raw_batch(7103, 3, 1501)
    hp = op.highpass_filter()
    p = Preprocessor(3, 1501, chan_map=np.array([2]), hp_filter=hp, do_CAR=False, device=DEV)
    X = p(torch.from_numpy(raw).to(DEV)).cpu().numpy()
    ref = op.filter_batch(torch.from_numpy(raw.T.astype(np.float64)), chan_map=torch.tensor([2]),
                          do_car=False, hp=hp.double()).numpy()
    assert np.abs(X - ref).max() <= 1e-5 * np.abs(ref).max()


def _car_expected(raw, cmap, invert, car):
    """The centring and common average reference in float32, as the kernel
    rounds them: the per-channel mean of the integer samples (exact sum in
    int64, divided in float64, rounded to float32, sign applied), one rounded
    difference, then the lower median of each sample over channels and one
    more rounded difference (torch.median of an even count is the lower one)."""
    x = raw[:, cmap].astype(np.float32)
    L, C = x.shape
    sign = np.float32(-1.0 if invert else 1.0)
    mean = (raw[:, cmap].astype(np.int64).sum(0).astype(np.float64) / L).astype(np.float32)
    v = sign * x - sign * mean
    if car:
        med = np.sort(v, axis=1)[:, (C - 1) // 2]
        v = v - med[:, None]
    return v.T


@pytest.mark.parametrize("C,L,kind,invert", [
    (384, 1100, "noise", False), (384, 1100, "noise", True), (63, 1037, "ties", False),
    (1000, 515, "noise", True), (2, 300, "noise", False), (1, 300, "noise", False),
    (384, 700, "crowded", False), (384, 700, "outliers", True)])
def test_car_median_exact(cuda_device, C, L, kind, invert):
    """The CAR output equals the float32 host computation bit for bit: bucketed
    median (noise, ties, outliers) and its radix-select fallback (a crowded
    median bucket: 300 of 384 channels equal)."""
    rng = np.random.default_rng(C * 1000 + L)
    n_bin = C + 3
    cmap = rng.permutation(n_bin)[:C]
    if kind == "ties":
        raw = rng.integers(-3, 4, (L, n_bin))
    else:
        raw = rng.normal(0, 40, (L, n_bin)) + rng.uniform(-300, 300, n_bin)
    if kind == "crowded":
        raw[:, cmap[:300]] = 17
    if kind == "outliers":
        hit = rng.random((L, n_bin)) < 0.05
        raw[hit] = rng.choice([-30000, 30000], hit.sum())
    raw = np.clip(np.round(raw), -32768, 32767).astype(np.int16)
    for car in (True, False):
        p = Preprocessor(n_bin, L, chan_map=cmap, do_CAR=car, invert_sign=invert, device=DEV)
        X = p(torch.from_numpy(raw).to(DEV)).cpu().numpy()
        assert p.status() == (_lib.KS_OK, False)
        np.testing.assert_array_equal(X, _car_expected(raw, cmap, invert, car))
