"""Golden vectors of the reference's Phy export, for the parts the matching
path produces.

Run from the repository root in a container that has the reference checkout,
after make_golden.py:

    python tests/golden/make_golden_phy.py path/to/reference

Takes the golden `extract` case (tests/golden/golden_extract.npz, recording
regenerated from its seed), adds near-duplicate spikes (copies of seeded
spikes 0-20 samples later, with the same template or another one, and their
features), and runs the reference's own ``io.save_to_phy``
(kilosort/io.py:248-470) on it into a temporary directory, with clusters =
templates and Wall = the templates' loadings in the clustering's layout
[K, C, P].  ``make_pc_features`` needs the clustering module's data and is
replaced by a stub that returns the features unchanged (its pc_features.npy
is not used); ``faiss`` (reached through kilosort/__init__) is replaced by an
empty module.  Stores the inputs and the files save_to_phy writes for spike
times, clusters, detection templates, positions, amplitudes, the kept-spike
mask, templates, their channel indices and the similarity, in
tests/golden/golden_phy.npz.
"""
import ast
import os
import sys
import tempfile
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from kilosort_b200 import synth  # noqa: E402

FILES = ["spike_times", "spike_templates", "spike_clusters", "spike_positions",
         "spike_detection_templates", "amplitudes", "kept_spikes", "templates",
         "templates_ind", "similar_templates"]


def reference_path():
    """The reference checkout: the first argument, else $KS_REFERENCE."""
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("KS_REFERENCE")
    if not ref:
        sys.exit(f"usage: python {os.path.basename(__file__)} PATH_TO_REFERENCE "
                 "(or set KS_REFERENCE)")
    return ref


def load_reference(path):
    sys.modules["faiss"] = types.ModuleType("faiss")
    pkg = types.ModuleType("kilosort")
    pkg.__path__ = [os.path.join(path, "kilosort")]
    sys.modules["kilosort"] = pkg
    from kilosort import io, template_matching
    io.make_pc_features = lambda ops, spike_templates, spike_clusters, tF: (
        tF, np.zeros((1, 1), np.uint32))
    return io, template_matching


def inputs(rec, g, seed=11):
    """st [N, 3] in time order with near-duplicates added, tF [N, nC, P]."""
    rng = np.random.default_rng(seed)
    st, tF = g["st"].copy(), g["tF"].copy()
    src = rng.choice(len(st), size=60, replace=False)
    add_st, add_tF = [], []
    for i, s in enumerate(src):
        row = st[s].copy()
        row[0] += int(rng.integers(0, 21))
        if i % 4 == 3:
            row[1] = (row[1] + 1) % rec.n_templates
        add_st.append(row)
        add_tF.append(tF[s])
    st = np.concatenate([st, np.array(add_st)])
    tF = np.concatenate([tF, np.array(add_tF)])
    order = np.argsort(st[:, 0], kind="stable")
    return st[order], tF[order]


if __name__ == "__main__":
    io, tm = load_reference(reference_path())
    g = np.load(os.path.join(HERE, "golden_extract.npz"))
    rec = synth.make_recording(**ast.literal_eval(str(g["seed_kwargs"])))
    st, tF = inputs(rec, g)
    U = torch.from_numpy(rec.U)
    W = torch.from_numpy(rec.wPCA)
    iCC, iCC_mask, iU, _ = tm.prepare_extract(rec.xc, rec.yc, U, 10, 100,
                                              device=torch.device("cpu"))
    C = rec.n_chan
    probe = dict(chanMap=np.arange(C), xc=rec.xc, yc=rec.yc, kcoords=np.zeros(C))
    ops = dict(iCC=iCC, iCC_mask=iCC_mask, iU=iU, xc=rec.xc, yc=rec.yc, wPCA=W, nt=rec.nt,
               fs=30000.0, duplicate_spike_bins=int(0.25 * 30000.0 / 1000), Wrot=torch.eye(C),
               settings=dict(acg_threshold=0.2, ccg_threshold=0.25, n_chan_bin=C,
                             fs=30000.0, filename="synthetic.bin"))
    clu = st[:, 1].astype(np.int32)
    Wall = U.transpose(1, 2).contiguous()
    out = {}
    with tempfile.TemporaryDirectory() as d:
        io.save_to_phy(st, clu, torch.from_numpy(tF), Wall, probe, ops, 0, results_dir=d)
        for name in FILES:
            out[name] = np.load(os.path.join(d, name + ".npy"))
    np.savez_compressed(os.path.join(HERE, "golden_phy.npz"), st=st, tF=tF, clu=clu,
                        dt=ops["duplicate_spike_bins"], **out)
    print(f"phy: {len(st)} spikes in, {int(out['kept_spikes'].sum())} kept, "
          f"templates {out['templates'].shape}")
