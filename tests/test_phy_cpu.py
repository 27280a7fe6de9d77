"""The oracle's duplicate removal and template waveforms against the
reference's own save_to_phy output (tests/golden/golden_phy.npz, made by
tests/golden/make_golden_phy.py): kept mask, spike arrays and templates."""
import ast

import numpy as np
import torch

from kilosort_b200 import synth
from oracle import postprocess as op
from tests.golden import make_golden_phy as mk

G = np.load(mk.__file__.replace("make_golden_phy.py", "golden_phy.npz"))


def test_remove_duplicates_matches_reference():
    st, clu, dt = G["st"], G["clu"], int(G["dt"])
    times, clusters, keep = op.remove_duplicates(st[:, 0].astype(np.int64), clu, dt)
    np.testing.assert_array_equal(keep, G["kept_spikes"])
    np.testing.assert_array_equal(times, G["spike_times"])
    np.testing.assert_array_equal(clusters, G["spike_clusters"])
    np.testing.assert_array_equal(st[:, 1].astype(np.int32)[keep], G["spike_detection_templates"])
    assert 0 < keep.sum() < len(keep)          # the case has duplicates to remove


def test_templates_match_reference():
    g = np.load(mk.__file__.replace("make_golden_phy.py", "golden_extract.npz"))
    rec = synth.make_recording(**ast.literal_eval(str(g["seed_kwargs"])))
    Wall = torch.from_numpy(rec.U).transpose(1, 2).contiguous()
    templates, ind = op.phy_templates(Wall, torch.from_numpy(rec.wPCA))
    np.testing.assert_array_equal(templates, G["templates"])
    np.testing.assert_array_equal(ind, G["templates_ind"])
