"""Golden vectors of the reference's output consumers of `extract`.

Run from the repository root in a container that has the reference checkout,
after make_golden.py:

    python tests/golden/make_golden_post.py path/to/reference

Loads the golden `extract` case (tests/golden/golden_extract.npz, its
recording regenerated from the stored seed), and runs the reference's
``postprocessing.compute_spike_positions`` (kilosort/postprocessing.py:33-62)
and the Phy-export amplitudes ``torch.norm(tF, dim=[-2, -1])``
(kilosort/io.py:353) on it; and the reference's template similarity
``CCG.similarity`` (kilosort/CCG.py:94-102, io.py:377) on that case's
templates in the clustering's layout (Wall = U transposed to [K, C, P]).  ``kilosort.clustering_qr`` (which needs faiss)
is replaced by an empty stub: compute_spike_positions does not use it.
Writes tests/golden/golden_post.npz.
"""
import ast
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from kilosort_b200 import synth  # noqa: E402


def reference_path():
    """The reference checkout: the first argument, else $KS_REFERENCE."""
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("KS_REFERENCE")
    if not ref:
        sys.exit(f"usage: python {os.path.basename(__file__)} PATH_TO_REFERENCE "
                 "(or set KS_REFERENCE)")
    return ref


def load_reference(path):
    pkg = types.ModuleType("kilosort")
    pkg.__path__ = [os.path.join(path, "kilosort")]
    sys.modules["kilosort"] = pkg
    stub = types.ModuleType("kilosort.clustering_qr")
    stub.xy_templates = None
    stub.get_data_cpu = None
    sys.modules["kilosort.clustering_qr"] = stub
    from kilosort import postprocessing, template_matching, CCG
    return postprocessing, template_matching, CCG


if __name__ == "__main__":
    ref = reference_path()
    post, tm, ccg = load_reference(ref)
    g = np.load(os.path.join(HERE, "golden_extract.npz"))
    rec = synth.make_recording(**ast.literal_eval(str(g["seed_kwargs"])))
    U = torch.from_numpy(rec.U)
    iCC, iCC_mask, iU, _ = tm.prepare_extract(rec.xc, rec.yc, U, 10, 100,
                                              device=torch.device("cpu"))
    ops = dict(iCC=iCC, iCC_mask=iCC_mask, iU=iU, xc=rec.xc, yc=rec.yc)
    st = g["st"]
    tF = torch.from_numpy(g["tF"])
    xs, ys = post.compute_spike_positions(st, tF, ops)
    amplitudes = torch.norm(tF, dim=[-2, -1]).cpu().numpy()
    Wall = U.transpose(1, 2).contiguous()
    sim = ccg.similarity(Wall, torch.from_numpy(rec.wPCA).contiguous(), nt=rec.nt)
    np.savez_compressed(os.path.join(HERE, "golden_post.npz"), xs=xs, ys=ys,
                        amplitudes=amplitudes, iCC_mask=iCC_mask.numpy(),
                        similarity=sim.astype(np.float32))
    print(f"post: {len(xs)} spikes")
