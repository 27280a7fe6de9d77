"""The universal-template detection oracle against the reference's own run()
(tests/golden/golden_detect.npz, made by tests/golden/make_golden_detect.py):
the derived geometry (nearest channels and template positions, size weights)
and every output (st, tF) are equal bit for bit."""
import ast

import numpy as np
import torch

from kilosort_b200 import synth
from oracle import detect as od
from tests.golden import make_golden_detect as mk

G = np.load(mk.__file__.replace("make_golden_detect.py", "golden_detect.npz"))


def golden_case():
    rec = synth.make_recording(**ast.literal_eval(str(G["seed_kwargs"])))
    ops = mk.make_ops(rec)
    return rec, ops


def test_geometry_matches_reference():
    rec, ops = golden_case()
    iC, iC2, weigh, ys, xs, dmin = od.setup(ops["xc"], ops["yc"], ops["kcoords"],
                                            ops["settings"], ops["max_channel_distance"])
    np.testing.assert_array_equal(iC.numpy(), G["iC"])
    np.testing.assert_array_equal(iC2.numpy(), G["iC2"])
    np.testing.assert_array_equal(weigh.numpy(), G["weigh"])
    np.testing.assert_array_equal(ys, G["ycup"])
    np.testing.assert_array_equal(xs, G["xcup"])
    assert dmin == float(G["dmin"])


def test_detection_matches_reference():
    rec, ops = golden_case()
    iC, iC2, weigh = (torch.from_numpy(G[k]) for k in ("iC", "iC2", "weigh"))
    batches = [torch.from_numpy(np.ascontiguousarray(rec.batch(b))) for b in range(rec.n_batches)]
    st, tF = od.run_batches(batches, torch.from_numpy(G["wTEMP"]), torch.from_numpy(G["wPCA"]),
                            iC, iC2, weigh, ops["yc"], rec.nt, ops["settings"]["nt0min"],
                            ops["Th_universal"], ops["batch_size"], ops["fs"])
    assert len(st) > 100
    np.testing.assert_array_equal(st, G["st"])
    np.testing.assert_array_equal(tF, G["tF"])
