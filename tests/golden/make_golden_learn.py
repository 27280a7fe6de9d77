"""Golden vectors of the reference's universal templates learned from data.

Run from the repository root in a container that has the reference checkout:

    python tests/golden/make_golden_learn.py path/to/reference

Runs the reference's own ``spikedetect.run`` with ``templates_from_data``
(kilosort/spikedetect.py:199-211, which calls ``extract_wPCA_wTEMP``,
:50-92: isolated single-channel peaks of every 25th batch, their unit-norm
snippets, a truncated SVD for wPCA and k-means for wTEMP) on CPU over a
seeded synthetic recording, and its ``extract_snippets`` (:33-48) on each
batch the learning step reads.  sklearn's TruncatedSVD and KMeans take their
randomness from numpy's global generator (random_state=None), which is
seeded here so the run can be repeated; the two estimators are wrapped only to
record the k-means inertia and the singular values they reach.  Writes
tests/golden/golden_learn.npz: the recording seed, the snippets, the learned
wPCA and wTEMP, those two figures, and run()'s outputs (st, tF) and geometry
(iC, iC2).
"""
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from kilosort_b200 import synth  # noqa: E402
import make_golden_detect as mk  # noqa: E402

SEED = dict(seed=9101, n_chan=64, probe="np1", n_templates=40,
            batch_lengths=[60000] * 26, rate_hz=(3.0, 8.0), amp_sd=(8.0, 16.0))
SETTINGS = dict(mk.SETTINGS, templates_from_data=True, Th_single_ch=6.0)
NSKIP = 25


def reference_path():
    """The reference checkout: the first argument, else $KS_REFERENCE."""
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("KS_REFERENCE")
    if not ref:
        sys.exit(f"usage: python {os.path.basename(__file__)} PATH_TO_REFERENCE "
                 "(or set KS_REFERENCE)")
    return ref


def make_ops(rec):
    ops = mk.make_ops(rec)
    ops["settings"] = dict(SETTINGS)
    ops["nt0min"] = SETTINGS["nt0min"]
    return ops


if __name__ == "__main__":
    sd = mk.load_reference(reference_path())
    rec = synth.make_recording(**SEED)
    ops = make_ops(rec)
    bfile = synth.SyntheticBinary(rec, device="cpu")
    cpu = torch.device("cpu")
    clips = []
    for j in range(0, bfile.n_batches, NSKIP):
        X = bfile.padded_batch_to_torch(j, ops)
        clips.append(sd.extract_snippets(X, nt=rec.nt, twav_min=ops["nt0min"],
                                         Th_single_ch=SETTINGS["Th_single_ch"],
                                         device=cpu).numpy())
    clips = np.concatenate(clips)
    # record the fitted estimators' objective values as the reference computes them
    fitted = {}

    class KMeans(sd.KMeans):
        def fit(self, X, *args, **kwargs):
            out = super().fit(X, *args, **kwargs)
            fitted["kmeans_inertia"] = float(self.inertia_)
            return out

    class TruncatedSVD(sd.TruncatedSVD):
        def fit(self, X, *args, **kwargs):
            out = super().fit(X, *args, **kwargs)
            fitted["svd_singular_values"] = self.singular_values_.copy()
            return out

    sd.KMeans, sd.TruncatedSVD = KMeans, TruncatedSVD
    np.random.seed(0)
    st, tF, ops = sd.run(ops, bfile, device=cpu)
    np.savez_compressed(
        os.path.join(HERE, "golden_learn.npz"), seed_kwargs=repr(SEED), clips=clips,
        wPCA=ops["wPCA"].numpy(), wTEMP=ops["wTEMP"].numpy(), st=st, tF=tF,
        iC=ops["iC"].numpy(), iC2=ops["iC2"].numpy(), **fitted)
    print(f"learn: {len(clips)} snippets, {len(st)} spikes, "
          f"{ops['iC'].shape[1]} template positions")
