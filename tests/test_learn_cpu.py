"""The oracle of the learned universal templates against the reference
(tests/golden/golden_learn.npz, made by tests/golden/make_golden_learn.py):
the snippets of the batches the learning step reads, exactly; the exact SVD
basis against the reference's randomized one where the singular values are
well apart, and in the energy it captures."""
import ast

import numpy as np
import torch

from kilosort_b200 import synth
from oracle import detect as od
from tests.golden import make_golden_learn as mk

G = np.load(mk.__file__.replace("make_golden_learn.py", "golden_learn.npz"))


def _clips():
    rec = synth.make_recording(**ast.literal_eval(str(G["seed_kwargs"])))
    out = []
    for j in range(0, rec.n_batches, mk.NSKIP):
        X = torch.from_numpy(np.ascontiguousarray(rec.batch(j)))
        out.append(od.extract_snippets(X, rec.nt, mk.SETTINGS["nt0min"],
                                       mk.SETTINGS["Th_single_ch"]).numpy())
    return np.concatenate(out)


def test_snippets_match_reference():
    clips = _clips()
    assert clips.shape == G["clips"].shape and len(clips) > 100
    np.testing.assert_array_equal(clips, G["clips"])


def test_svd_basis_against_reference():
    basis = od.svd_basis(G["clips"], 6)
    ref = G["wPCA"].astype(np.float64)
    # the leading components (singular values 18.1, 3.10, 2.52: well apart)
    assert np.abs(basis[:3] - ref[:3]).max() < 1e-4
    # the captured energy of the whole basis
    x = G["clips"].astype(np.float64)
    x /= np.sqrt((x ** 2).sum(1, keepdims=True))
    g = x.T @ x
    e_ours = np.trace(basis @ g @ basis.T)
    e_ref = np.trace(ref @ g @ ref.T)
    assert e_ours >= e_ref * (1 - 1e-6)
    assert abs(e_ours - e_ref) <= 1e-4 * e_ref
