"""The CPU oracle reproduces the reference's own outputs bit for bit.

Golden vectors come from running the reference's `prepare_matching`,
`run_matching`, `prepare_extract` and `extract` (tests/golden/make_golden.py).
"""
import ast
import os

import numpy as np
import pytest
import torch

from oracle import matching as om
from tests import golden_util as gu


@pytest.mark.parametrize("name", gu.CASES)
def test_run_matching_bit_exact(name):
    g = gu.load(name)
    rec, X, U, W = gu.case_inputs(g)
    Ut, Wt = torch.from_numpy(U), torch.from_numpy(W)
    ops = dict(Th_learned=float(g["Th"]), nt=int(g["nt"]),
               max_peels=int(g["max_peels"]), wPCA=Wt)
    ctc = om.prepare_matching(ops, Ut)
    assert gu.sha(ctc.numpy()) == str(g["ctc_sha"])
    st, amps, th, Xres = om.run_matching(ops, torch.from_numpy(X), Ut, ctc)
    np.testing.assert_array_equal(st.numpy(), g["st"])
    np.testing.assert_array_equal(amps.numpy(), g["amps"])
    np.testing.assert_array_equal(th.numpy(), g["th_amps"])
    assert gu.sha(Xres.numpy()) == str(g["xres_sha"])


def test_stored_inputs_match_generator():
    g = gu.load("tiny")
    rec, X, U, W = gu.case_inputs(g)
    np.testing.assert_array_equal(g["X"], X)
    np.testing.assert_array_equal(g["U"], U)
    np.testing.assert_array_equal(g["W"], W)


def test_prepare_extract_bit_exact():
    g = gu.load("small")
    rec, X, U, W = gu.case_inputs(g)
    iCC, mask, iU, Ucc = om.prepare_extract(g["xc"], g["yc"], torch.from_numpy(U),
                                            10, 100)
    np.testing.assert_array_equal(iCC.numpy(), g["iCC"])
    np.testing.assert_array_equal(mask.numpy(), g["iCC_mask"])
    np.testing.assert_array_equal(iU.numpy(), g["iU"])
    np.testing.assert_array_equal(Ucc.numpy(), g["Ucc"])


def test_extract_features_bit_exact():
    """Oracle batch loop (matching + features + time shift) equals `extract`."""
    from kilosort_b200 import synth
    g = gu.load("extract")
    kw = ast.literal_eval(str(g["seed_kwargs"]))
    rec = synth.make_recording(**kw)
    assert gu.sha(rec.signal) == str(g["signal_sha"])
    U = torch.from_numpy(rec.U)
    W = torch.from_numpy(rec.wPCA)
    nt, nt0min, NT = 61, 20, 3000
    ops = dict(Th_learned=8.0, nt=nt, max_peels=100, wPCA=W)
    iCC, _, iU, Ucc = om.prepare_extract(rec.xc, rec.yc, U, 10, 100)
    ctc = om.prepare_matching(ops, U)
    rows, feats = [], []
    for b in range(rec.n_batches):
        X = torch.from_numpy(np.ascontiguousarray(rec.batch(b)))
        st, amps, th, Xres = om.run_matching(ops, X, U, ctc)
        f = om.spike_features(Xres, st, amps, W, iCC, iU, Ucc, nt)
        if b == 0:
            keep = (st[:, 0] - nt - nt // 2 + nt0min) >= 0
            st, f, th = st[keep], f[:, keep], th[keep]
        t = (st[:, 0].double() - nt + b * NT).numpy() - nt // 2 + nt0min
        rows.append(np.stack([t, st[:, 1].double().numpy(),
                              th.numpy().squeeze(1).astype(np.float64)], 1))
        feats.append(f.transpose(0, 1))
    st_all = np.concatenate(rows)
    tF = torch.cat(feats)
    order = np.argsort(st_all[:, 0])
    np.testing.assert_array_equal(st_all[order], g["st"])
    np.testing.assert_array_equal(tF[order].numpy(), g["tF"])


def test_output_consumers_bit_exact():
    """Oracle positions, amplitudes and template similarity equal the reference's
    on the golden extract case."""
    from kilosort_b200 import synth
    from oracle import postprocess as op
    g = gu.load("extract")
    post = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_post.npz"))
    kw = ast.literal_eval(str(g["seed_kwargs"]))
    rec = synth.make_recording(**kw)
    iCC, mask, iU, _ = om.prepare_extract(rec.xc, rec.yc, torch.from_numpy(rec.U), 10, 100)
    np.testing.assert_array_equal(mask.numpy(), post["iCC_mask"])
    xs, ys = op.spike_positions(g["st"], torch.from_numpy(g["tF"]), iCC, mask, iU, rec.xc, rec.yc)
    np.testing.assert_array_equal(xs, post["xs"])
    np.testing.assert_array_equal(ys, post["ys"])
    np.testing.assert_array_equal(op.amplitudes(torch.from_numpy(g["tF"])), post["amplitudes"])
    Wall = torch.from_numpy(rec.U).transpose(1, 2).contiguous()
    np.testing.assert_array_equal(op.similarity(Wall, torch.from_numpy(rec.wPCA), rec.nt),
                                  post["similarity"])
