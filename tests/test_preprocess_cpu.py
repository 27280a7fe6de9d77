"""The batch preprocessing oracle against the reference's own filter (CPU).

tests/golden/golden_pre.npz holds the output of the reference's
BinaryFiltered.filter (kilosort/io.py:994-1026) on seeded raw batches; the
oracle restates it with the same PyTorch operations (bit-for-bit equal here),
and its float64 circular-correlation form with the 1023 centre taps of the
high-pass and the centre offset of odd batch lengths (the form the device
computes) agrees to 1e-5 of the batch maximum
(the reference's own float32 FFT error, and the filter's tail beyond 511
samples, stay far below that).
"""
import hashlib

import numpy as np
import pytest
import torch

from kilosort_b200 import synth
from oracle import preprocess as op
from tests.golden import make_golden_pre as mk

G = np.load(mk.__file__.replace("make_golden_pre.py", "golden_pre.npz"))


def _case(name):
    seed, L, inv, car, use_hp, use_w, shift = G[f"{name}_params"]
    raw = synth.raw_batch(int(seed), int(G["n_chan_bin"]), int(L))
    assert hashlib.sha256(raw.tobytes()).hexdigest()[:16] == str(G[f"{name}_raw_sha"])
    kw = dict(chan_map=torch.from_numpy(G["chan_map"]), invert_sign=bool(inv),
              do_car=bool(car), artifact_threshold=float(G[f"{name}_thr"]),
              whiten=torch.from_numpy(G[f"{name}_W"]) if use_w else None)
    drift = None
    if shift >= 0:
        drift = op.drift_matrix(G[f"{name}_xc"], G[f"{name}_yc"], float(shift)).float()
    return raw, bool(use_hp), drift, kw


@pytest.mark.parametrize("name", list(mk.CASES))
def test_oracle_equals_reference_filter(name):
    raw, use_hp, drift, kw = _case(name)
    hp = op.highpass_filter() if use_hp else None
    X = torch.from_numpy(raw.T.astype(np.float32))
    Y = op.filter_batch(X, hp=hp, drift=drift, **kw).numpy()
    np.testing.assert_array_equal(Y, G[f"{name}_out"])


@pytest.mark.parametrize("name", list(mk.CASES))
def test_centre_tap_correlation_matches_fft_form(name):
    raw, use_hp, drift, kw = _case(name)
    taps, centre = op.centre_taps(op.highpass_filter(), raw.shape[0]) if use_hp else (None, 0)
    X = torch.from_numpy(raw.T.astype(np.float32))
    Y = op.filter_batch_taps(X, taps, centre, drift=drift, **kw).numpy()
    ref = G[f"{name}_out"]
    scale = max(np.abs(ref).max(), 1.0)
    assert np.abs(Y - ref).max() <= 1e-5 * scale, (name, np.abs(Y - ref).max(), scale)


def test_highpass_taps_are_symmetric_and_decay():
    hp = op.highpass_filter()
    taps, centre = op.centre_taps(hp, 60122)
    assert len(taps) == 1023 and centre == 511
    assert np.array_equal(taps, taps[::-1])
    assert abs(taps[511] - float(hp[15061])) == 0.0
    assert np.abs(taps[:8]).max() < 1e-9 * taps.max()
    # odd batch lengths: the cropped (L < 30122) filter's centre sits one
    # sample past L//2, the padded (L > 30122) one at L//2
    assert op.centre_taps(hp, 1101)[1] == 511 - 1
    assert op.centre_taps(hp, 40001)[1] == 511
    # short batches keep only the taps the cropped filter holds
    taps, centre = op.centre_taps(hp, 600)
    assert len(taps) == 599 and centre == 299
