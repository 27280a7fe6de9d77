"""The Phy-export arrays on the device (ks_remove_duplicates,
ks_phy_templates, ks_spike_positions, ks_similarity through
postprocess.phy_arrays) against the reference's own save_to_phy output
(tests/golden/golden_phy.npz), and the duplicate removal against the oracle
on seeded inputs in arbitrary order (many clusters, ties, equal times).

Tolerances: integer arrays and the kept mask exactly; templates within 1e-6
of the largest (products summed over the components in order, as the
reference); positions within 1e-4 um, amplitudes 1e-6 relative, similarity
1e-5 (as the other output-consumer tests).
"""
import ast

import numpy as np
import pytest
import torch

from kilosort_b200 import postprocess as pp
from kilosort_b200 import synth
from oracle import matching as om
from oracle import postprocess as op
from tests.golden import make_golden_phy as mk

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
G = np.load(mk.__file__.replace("make_golden_phy.py", "golden_phy.npz"))


def test_phy_arrays_match_reference_save_to_phy(cuda_device):
    g = np.load(mk.__file__.replace("make_golden_phy.py", "golden_extract.npz"))
    rec = synth.make_recording(**ast.literal_eval(str(g["seed_kwargs"])))
    U = torch.from_numpy(rec.U)
    iCC, mask, iU, _ = om.prepare_extract(rec.xc, rec.yc, U, 10, 100)
    ops = dict(iCC=iCC.to(DEV), iCC_mask=mask.to(DEV), iU=iU.to(DEV), xc=rec.xc, yc=rec.yc,
               wPCA=torch.from_numpy(rec.wPCA).to(DEV), nt=rec.nt,
               duplicate_spike_bins=int(G["dt"]))
    Wall = U.transpose(1, 2).contiguous().to(DEV)
    out = pp.phy_arrays(G["st"], G["clu"], G["tF"], Wall, ops, imin=0)
    for name in ("spike_times", "spike_templates", "spike_clusters",
                 "spike_detection_templates", "kept_spikes", "templates_ind"):
        np.testing.assert_array_equal(out[name], G[name], err_msg=name)
        assert out[name].dtype == G[name].dtype, name
    t = G["templates"]
    assert out["templates"].shape == t.shape
    assert np.abs(out["templates"] - t).max() <= 1e-6 * np.abs(t).max()
    np.testing.assert_allclose(out["spike_positions"], G["spike_positions"], rtol=0, atol=1e-4)
    np.testing.assert_allclose(out["amplitudes"], G["amplitudes"], rtol=1e-6)
    np.testing.assert_allclose(out["similar_templates"], G["similar_templates"], rtol=0,
                               atol=1e-5)


@pytest.mark.parametrize("seed,n,k,dt", [(1, 20000, 50, 7), (2, 5000, 3, 30), (3, 1, 1, 7),
                                         (4, 30000, 2000, 0)])
def test_remove_duplicates_matches_oracle_any_order(cuda_device, seed, n, k, dt):
    rng = np.random.default_rng(seed)
    times = rng.integers(0, 10 * n + 10, size=n).astype(np.int64)
    times[rng.random(n) < 0.1] = 17                       # equal times across clusters
    clusters = rng.integers(0, k, size=n).astype(np.int32)
    if seed % 2:
        order = np.argsort(times, kind="stable")          # time order, as save_to_phy
        times, clusters = times[order], clusters[order]
    t_r, c_r, keep_r = op.remove_duplicates(times, clusters, dt)
    t, c, keep = pp.remove_duplicates(times, clusters, dt, device=DEV)
    np.testing.assert_array_equal(keep, keep_r)
    np.testing.assert_array_equal(t, t_r)
    np.testing.assert_array_equal(c, c_r)


def test_remove_duplicates_empty(cuda_device):
    t, c, keep = pp.remove_duplicates(np.zeros(0, np.int64), np.zeros(0, np.int32), 7,
                                      device=DEV)
    assert t.size == c.size == keep.size == 0
