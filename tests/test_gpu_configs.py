"""Parity at the shapes of the uneven multi-recording workload and of the long
dense stream, against the oracle.

* Uneven batches (C/K = 96/150, 384/600, 384/1000; lengths drawn from
  U[8000, 60000] with a short tail batch per recording, the generator of the
  uneven benchmark with two batches per recording): every batch of one
  ks_match_batches call is compared with the oracle's run_matching on it.
* Dense stream (C=384, K=2000, 60000-sample batches, amplitudes 5-40 sd,
  1-30 Hz, int16 on the host): the StreamMatcher's spikes of each batch are
  compared with the oracle's run_matching on the same whitened batch.

The oracle restates kilosort/template_matching.py:170-244 with the
reference's torch ops and is pinned bit for bit to the reference on the CPU
(test_oracle_golden.py).  At these sizes (up to 2000 templates, ~60000 spikes
per batch) it runs on the GPU, with TF32 off so its convolution and
contractions are FP32, as the reference's own op sequence on a GPU would.
Bar: >= 99.5 % exact (time, template) agreement per batch; amplitude relative
error <= 1e-4 with the FP32 projection and <= 1e-3 with the split-BF16 one,
at the 99.9th percentile of the matched spikes and as the maximum over the
matched spikes farther than 4*nt samples from any spike that only one side
found (a spike found by one side alone -- a near-threshold flip -- changes the
subtractions and so the amplitudes of its neighbours).
"""
import numpy as np
import pytest
import torch

import kilosort_b200 as kb
from kilosort_b200 import synth
from kilosort_b200.batched import Recording, match_batches
from kilosort_b200.stream import StreamMatcher, Whitener, batch_windows, padded_raw_window
from oracle import matching as om
from tests.parity_util import agreement

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
AMP_TOL = {"fp32": 1e-4, "bf16x3": 1e-3}


class _NoTF32:
    def __enter__(self):
        self.flags = (torch.backends.cudnn.allow_tf32, torch.backends.cuda.matmul.allow_tf32)
        torch.backends.cudnn.allow_tf32 = False
        torch.backends.cuda.matmul.allow_tf32 = False

    def __exit__(self, *a):
        torch.backends.cudnn.allow_tf32, torch.backends.cuda.matmul.allow_tf32 = self.flags


def _oracle(ops, X, U, ctc):
    with _NoTF32():
        st, amps, _, _ = om.run_matching(ops, X, U, ctc)
    return st.cpu().numpy(), amps.cpu().numpy()


def _isolated_amp_error(st, amps, st_r, amps_r, guard):
    """Largest amplitude relative error over matched (time, template) pairs
    farther than `guard` samples from every spike that only one list has: a
    spike found by one side alone changes the subtractions around it, so its
    neighbours' amplitudes legitimately differ."""
    key = lambda s: s[:, 0].astype(np.int64) * 1_000_003 + s[:, 1].astype(np.int64)
    ka, kr = key(st), key(st_r)
    odd = np.concatenate([st[~np.isin(ka, kr), 0], st_r[~np.isin(kr, ka), 0]])
    ia = {}                      # key -> our indices in order (a pair may repeat)
    for i, k in enumerate(ka.tolist()):
        ia.setdefault(k, []).append(i)
    err = 0.0
    for j, k in enumerate(kr.tolist()):
        occ = ia.get(k)
        if not occ:
            continue
        i = occ.pop(0)
        t = st_r[j, 0]
        if len(odd) and np.min(np.abs(odd - t)) <= guard:
            continue
        ref = float(np.asarray(amps_r).reshape(-1)[j])
        err = max(err, abs(float(np.asarray(amps).reshape(-1)[i]) - ref) / max(abs(ref), 1e-30))
    return err


def _check(st, amps, st_r, amps_r, projection, what, nt=61):
    a = agreement(st, st_r, amps, amps_r)
    assert a["n_r"] > 0, what
    assert a["agreement"] >= 0.995, (what, a)
    assert a["amp_rel_p999"] <= AMP_TOL[projection], (what, a)
    iso = _isolated_amp_error(np.asarray(st), amps, np.asarray(st_r), amps_r, 4 * nt)
    assert iso <= AMP_TOL[projection], (what, iso, a)
    return a


@pytest.mark.parametrize("projection", ["fp32", "bf16x3"])
def test_uneven_recordings_vs_oracle(cuda_device, projection):
    recs = synth.uneven_recordings(seed=1003, n_batches_total=6)
    assert [(r.n_chan, r.n_templates) for r in recs] == [(96, 150), (384, 600), (384, 1000)]
    mrecs, ops_l, items = [], [], []
    for i, r in enumerate(recs):
        U = torch.from_numpy(r.U).to(DEV)
        W = torch.from_numpy(r.wPCA).to(DEV)
        ops = dict(Th_learned=8.0, nt=r.nt, max_peels=100, wPCA=W)
        with _NoTF32():
            ctc = om.prepare_matching(ops, U)
        mrecs.append(Recording.from_ops(ops, U, ctc))
        ops_l.append((ops, U, ctc))
        for b in range(r.n_batches):
            items.append((torch.from_numpy(np.ascontiguousarray(r.batch(b))).to(DEV), i))
    lengths = sorted(X.shape[1] - 2 * 61 for X, _ in items)
    assert lengths[0] < 8000 <= lengths[-1] <= 60000      # a tail batch and a long one
    res = match_batches(mrecs, items, projection=projection, teams=3)
    for (X, r), (st, amps, _, _) in zip(items, res):
        ops, U, ctc = ops_l[r]
        st_r, amps_r = _oracle(ops, X, U, ctc)
        _check(st.cpu().numpy(), amps.cpu().numpy(), st_r, amps_r, projection,
               f"recording {r}, L={X.shape[1]}")


def _mixing(C, seed=0):
    rng = np.random.default_rng(seed)
    M = np.eye(C)
    for d in (1, 2):
        v = 0.25 / d * (1 + 0.2 * rng.standard_normal(C - d))
        M += np.diag(v, d) + np.diag(v, -d)
    return M


def test_dense_stream_k2000_vs_oracle(cuda_device):
    NT, nb = 60000, 2
    c = dict(synth.CONFIGS[5])
    c.pop("n_batches")
    rec = synth.make_recording(1005, batch_lengths=[NT] * nb, **c)
    assert (rec.n_chan, rec.n_templates) == (384, 2000)
    M = _mixing(rec.n_chan, 1005)
    raw = np.clip(np.round(200.0 * (M @ rec.signal.astype(np.float64))).T, -32768, 32767)
    raw = raw.astype(np.int16)
    Wrot = torch.from_numpy(np.linalg.inv(M)).float()
    scale = 1.0 / 200.0
    U = torch.from_numpy(rec.U).to(DEV)
    W = torch.from_numpy(rec.wPCA).to(DEV)
    nt = rec.nt
    ops = dict(Th_learned=8.0, nt=nt, max_peels=100, wPCA=W)
    sm = StreamMatcher(raw, Wrot, scale, ops, U, NT=NT, group=nb, teams=2)
    times, templ, amps, bidx = sm.run()
    sm.close()
    # the oracle on the same whitened batches
    w = Whitener(Wrot, scale, NT + 2 * nt, DEV)
    with _NoTF32():
        ctc = om.prepare_matching(ops, U)
    n_total = 0
    for b in range(len(batch_windows(raw.shape[0], NT, nt))):
        win = padded_raw_window(raw, b, NT, nt, np.empty((NT + 2 * nt, raw.shape[1]), np.int16))
        X = torch.empty((raw.shape[1], NT + 2 * nt), device=DEV)
        w(torch.from_numpy(win).to(DEV), X)
        st_r, amps_r = _oracle(ops, X, U, ctc)
        sel = bidx == b
        st = np.stack([times[sel] + nt - b * NT, templ[sel]], axis=1)
        a = _check(st, amps[sel], st_r, amps_r, "bf16x3", f"batch {b}")
        n_total += a["n_r"]
    assert n_total > 30000          # a dense batch: tens of thousands of spikes
