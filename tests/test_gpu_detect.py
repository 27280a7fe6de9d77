"""Universal-template detection on the device (ks_detect) against the
reference's own run() (tests/golden/golden_detect.npz) and the oracle.

Tolerances: the detected (batch, position, sample) set agrees with the
reference's at >= 99.5 % (its sums over channels run in another order, so a
peak within rounding of Th_universal or of a neighbour's value may flip);
on matched spikes the signed index is equal, amplitudes within 1e-5
relative, y within 1e-3 um, features within 1e-5 of the largest.
"""
import ast

import numpy as np
import pytest
import torch

from kilosort_b200 import _lib, synth
from kilosort_b200 import spikedetect as sd
from oracle import detect as od
from tests.golden import make_golden_detect as mk

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
G = np.load(mk.__file__.replace("make_golden_detect.py", "golden_detect.npz"))


def _ops(rec):
    ops = mk.make_ops(rec)
    ops["wTEMP"] = torch.from_numpy(G["wTEMP"])
    ops["wPCA"] = torch.from_numpy(G["wPCA"])
    return ops


def _compare(st, tF, st_r, tF_r):
    key = lambda s: {(int(b), int(f), round(t * 30000.0)): i
                     for i, (t, f, b) in enumerate(zip(s[:, 0], s[:, 5], s[:, 4]))}
    a, r = key(st), key(st_r)
    both = sorted(set(a) & set(r))
    agree = min(len(both) / max(len(r), 1), len(both) / max(len(a), 1))
    assert agree >= 0.995, (agree, len(a), len(r))
    ia = np.array([a[k] for k in both])
    ir = np.array([r[k] for k in both])
    np.testing.assert_array_equal(st[ia, 3], st_r[ir, 3])
    np.testing.assert_allclose(st[ia, 2], st_r[ir, 2], rtol=1e-5)
    np.testing.assert_allclose(st[ia, 1], st_r[ir, 1], rtol=0, atol=1e-3)
    scale = np.abs(tF_r).max()
    assert np.abs(tF[ia] - tF_r[ir]).max() <= 1e-5 * scale
    return len(both)


def test_run_matches_reference(cuda_device, tmp_path, monkeypatch):
    # the built-in templates branch (templates_from_data off): run() reads
    # wTEMP.npz where the reference keeps its download
    np.savez(tmp_path / "wTEMP.npz", wTEMP=G["wTEMP"], wPCA=G["wPCA"])
    monkeypatch.setenv("KILOSORT_LOCAL_DOWNLOADS_PATH", str(tmp_path))
    rec = synth.make_recording(**ast.literal_eval(str(G["seed_kwargs"])))
    ops = mk.make_ops(rec)
    st, tF, ops = sd.run(ops, synth.SyntheticBinary(rec, device=DEV), device=DEV)
    np.testing.assert_array_equal(ops["wTEMP"].cpu().numpy(), G["wTEMP"])
    np.testing.assert_array_equal(ops["iC"].cpu().numpy(), G["iC"])
    np.testing.assert_array_equal(ops["iC2"].cpu().numpy(), G["iC2"])
    assert _compare(st, tF, G["st"], G["tF"]) > 100


def test_np1_scale_batch_matches_oracle(cuda_device):
    rec = synth.make_recording(9002, n_chan=384, probe="np1", n_templates=200,
                               batch_lengths=[15000], rate_hz=(5.0, 20.0), amp_sd=(10.0, 30.0))
    ops = _ops(rec)
    iC, iC2, weigh = sd.geometry(ops, device=DEV)
    assert iC.shape[1] > 1000
    X = torch.from_numpy(np.ascontiguousarray(rec.batch(0)))
    det = sd.Detector(ops, iC, iC2, weigh, DEV)
    xy, imax, amp, adist, yct, tF = det(X.to(DEV))
    st, tF_all = od.run_batches([X], ops["wTEMP"], ops["wPCA"], iC.cpu(), iC2.cpu(),
                                weigh.cpu(), ops["yc"], rec.nt, ops["settings"]["nt0min"],
                                ops["Th_universal"], ops["batch_size"], ops["fs"])
    mine = np.zeros((len(xy), 6))
    xy_h = xy.cpu().numpy()
    mine[:, 0] = (xy_h[:, 1] - rec.nt) / ops["fs"]
    mine[:, 1] = yct.cpu().numpy()
    mine[:, 2] = amp.cpu().numpy()
    mine[:, 3] = imax.cpu().numpy()
    mine[:, 5] = xy_h[:, 0]
    assert _compare(mine, tF.cpu().numpy(), st, tF_all) > 300


def test_small_capacity_retries_to_the_same_result(cuda_device):
    rec = synth.make_recording(**ast.literal_eval(str(G["seed_kwargs"])))
    ops = _ops(rec)
    iC, iC2, weigh = sd.geometry(ops, device=DEV)
    X = torch.from_numpy(np.ascontiguousarray(rec.batch(0))).to(DEV)
    full = sd.Detector(ops, iC, iC2, weigh, DEV)(X)
    small = sd.Detector(ops, iC, iC2, weigh, DEV, capacity=5)(X)
    assert len(full[0]) > 5
    for a, b in zip(full, small):
        assert torch.equal(a, b)


def test_bad_channel_index_is_reported(cuda_device):
    rec = synth.make_recording(**ast.literal_eval(str(G["seed_kwargs"])))
    ops = _ops(rec)
    iC, iC2, weigh = sd.geometry(ops, device=DEV)
    iC = iC.clone()
    iC[0, 0] = rec.n_chan + 3
    X = torch.from_numpy(np.ascontiguousarray(rec.batch(0))).to(DEV)
    with pytest.raises(_lib.KilosortB200Error):
        sd.Detector(ops, iC, iC2, weigh, DEV)(X)


def test_zero_batch_has_no_spikes(cuda_device):
    rec = synth.make_recording(**ast.literal_eval(str(G["seed_kwargs"])))
    ops = _ops(rec)
    iC, iC2, weigh = sd.geometry(ops, device=DEV)
    X = torch.zeros((rec.n_chan, 3122), device=DEV)
    xy, imax, amp, adist, yct, tF = sd.Detector(ops, iC, iC2, weigh, DEV)(X)
    assert len(xy) == len(imax) == len(amp) == len(yct) == len(tF) == 0
    assert adist.shape == (iC.shape[0], 0)


def test_run_without_templates_file_raises(cuda_device, tmp_path, monkeypatch):
    monkeypatch.setenv("KILOSORT_LOCAL_DOWNLOADS_PATH", str(tmp_path))
    rec = synth.make_recording(**ast.literal_eval(str(G["seed_kwargs"])))
    with pytest.raises(FileNotFoundError):
        sd.run(mk.make_ops(rec), synth.SyntheticBinary(rec, device=DEV), device=DEV)
