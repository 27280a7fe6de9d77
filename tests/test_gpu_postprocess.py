"""Spike positions and amplitudes on the GPU (ks_spike_positions) against the
reference's own outputs on the golden extract case (positions within 1e-4 um,
amplitudes within 1e-6 relative: the kernel's norms sum in another order), and
the template similarity (ks_similarity) against the reference's CCG.similarity
(within 1e-5 of the largest entry: FP32 sums in another order), also at
C=384 / K=600 against the oracle."""
import ast
import os

import numpy as np
import pytest
import torch

import kilosort_b200 as kb
from kilosort_b200 import postprocess, synth
from oracle import postprocess as op
from tests import golden_util as gu

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _ops(rec):
    iCC, mask, iU, _ = kb.prepare_extract(rec.xc, rec.yc, torch.from_numpy(rec.U).to(DEV), 10,
                                          100, device=DEV)
    return dict(iCC=iCC, iCC_mask=mask, iU=iU, xc=rec.xc, yc=rec.yc)


def test_positions_and_amplitudes_match_reference(cuda_device):
    g = gu.load("extract")
    post = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_post.npz"))
    rec = synth.make_recording(**ast.literal_eval(str(g["seed_kwargs"])))
    ops = _ops(rec)
    xs, ys = postprocess.compute_spike_positions(g["st"], torch.from_numpy(g["tF"]), ops)
    np.testing.assert_allclose(xs, post["xs"], rtol=0, atol=1e-4)
    np.testing.assert_allclose(ys, post["ys"], rtol=0, atol=1e-4)
    amps = postprocess.spike_amplitudes(torch.from_numpy(g["tF"]), ops)
    np.testing.assert_allclose(amps, post["amplitudes"], rtol=1e-6)


def test_positions_after_gpu_extract(cuda_device):
    g = gu.load("extract")
    rec = synth.make_recording(**ast.literal_eval(str(g["seed_kwargs"])))
    bfile = synth.SyntheticBinary(rec, device=DEV)
    ops = dict(Th_learned=8.0, nt=61, max_peels=100, wPCA=torch.from_numpy(rec.wPCA).to(DEV),
               nt0min=20, batch_size=3000, xc=rec.xc, yc=rec.yc,
               settings=dict(nearest_chans=10, position_limit=100, n_pcs=6))
    st, tF, ops = kb.extract(ops, bfile, torch.from_numpy(rec.U).to(DEV), device=DEV)
    xs, ys = postprocess.compute_spike_positions(st, tF, ops)
    xr, yr = op.spike_positions(st, tF, ops["iCC"].cpu(), ops["iCC_mask"].cpu(),
                                ops["iU"].cpu(), rec.xc, rec.yc)
    np.testing.assert_allclose(xs, xr, rtol=0, atol=1e-4)
    np.testing.assert_allclose(ys, yr, rtol=0, atol=1e-4)


def test_bad_template_index_is_reported(cuda_device):
    g = gu.load("extract")
    rec = synth.make_recording(**ast.literal_eval(str(g["seed_kwargs"])))
    ops = _ops(rec)
    st = g["st"].copy()
    st[0, 1] = 10 ** 6
    with pytest.raises(kb._lib.KilosortB200Error):
        postprocess.compute_spike_positions(st, torch.from_numpy(g["tF"]), ops)


def test_similarity_matches_reference(cuda_device):
    g = gu.load("extract")
    post = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_post.npz"))
    rec = synth.make_recording(**ast.literal_eval(str(g["seed_kwargs"])))
    Wall = torch.from_numpy(rec.U).transpose(1, 2).contiguous().to(DEV)
    sim = postprocess.template_similarity(Wall, torch.from_numpy(rec.wPCA).to(DEV), rec.nt)
    ref = post["similarity"]
    assert np.abs(sim - ref).max() <= 1e-5 * np.abs(ref).max()


def test_similarity_cfg2_templates(cuda_device):
    rec = synth.config_recording(2, n_batches=1)
    Wall = torch.from_numpy(rec.U).transpose(1, 2).contiguous()
    W = torch.from_numpy(rec.wPCA)
    sim = postprocess.template_similarity(Wall.to(DEV), W.to(DEV), rec.nt)
    ref = op.similarity(Wall, W, rec.nt)
    assert sim.shape == (600, 600)
    assert np.abs(sim - ref).max() <= 1e-5 * np.abs(ref).max()
    # each template is most similar to itself (unit norm: about 1 at lag 0)
    assert np.all(np.abs(np.diag(sim) - 1) < 1e-3)


def test_similarity_single_template(cuda_device):
    rec = synth.make_recording(8301, n_chan=16, n_templates=1, batch_lengths=[3000])
    Wall = torch.from_numpy(rec.U).transpose(1, 2).contiguous()
    sim = postprocess.template_similarity(Wall.to(DEV), torch.from_numpy(rec.wPCA).to(DEV),
                                          rec.nt)
    ref = op.similarity(Wall, torch.from_numpy(rec.wPCA), rec.nt)
    assert sim.shape == (1, 1) and abs(sim[0, 0] - ref[0, 0]) <= 1e-5
