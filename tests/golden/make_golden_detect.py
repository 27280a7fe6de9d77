"""Golden vectors of the reference's universal-template spike detection.

Run from the repository root in a container that has the reference checkout:

    python tests/golden/make_golden_detect.py path/to/reference

Runs the reference's own ``spikedetect.run`` (kilosort/spikedetect.py:199-307:
template centres, nearest channels and templates, size weights, then per
batch ``template_match`` (:133-178), ``yweighted`` and the PC features) on
CPU over a seeded synthetic recording served by a batch source with the
duck type run() reads (``n_batches``, ``batch_downsampling``,
``padded_batch_to_torch``), with the reference's built-in universal
templates (kilosort/wTEMP.npz, read from the checkout instead of the
download cache).  ``faiss`` (reached through kilosort/__init__) is replaced
by an empty module.  Writes tests/golden/golden_detect.npz: the recording
seed, the templates, run()'s outputs (st, tF) and the geometry it derived
(iC, iC2, weigh, ycup, xcup).
"""
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from kilosort_b200 import synth  # noqa: E402

SEED = dict(seed=9001, n_chan=64, probe="np1", n_templates=30, batch_lengths=[3000, 3000],
            rate_hz=(20.0, 60.0), amp_sd=(10.0, 30.0))
SETTINGS = dict(nearest_chans=10, nearest_templates=100, min_template_size=10,
                template_sizes=5, dmin=None, dminx=32, n_templates=6, n_pcs=6, nt0min=20,
                templates_from_data=False)


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
    from kilosort import spikedetect
    wtemp = os.path.join(path, "kilosort", "wTEMP.npz")
    spikedetect.template_path = lambda basename="wTEMP.npz": wtemp
    return spikedetect


def make_ops(rec):
    return dict(settings=dict(SETTINGS), xc=rec.xc.astype(np.float32),
                yc=rec.yc.astype(np.float32), kcoords=np.zeros(rec.n_chan, np.float32),
                Nbatches=rec.n_batches, nt=rec.nt, batch_size=int(rec.batch_lengths[0]),
                fs=30000.0, Th_universal=9.0, max_channel_distance=32.0)


if __name__ == "__main__":
    ref = reference_path()
    sd = load_reference(ref)
    rec = synth.make_recording(**SEED)
    ops = make_ops(rec)
    bfile = synth.SyntheticBinary(rec, device="cpu")
    st, tF, ops = sd.run(ops, bfile, device=torch.device("cpu"))
    w = np.load(os.path.join(ref, "kilosort", "wTEMP.npz"))
    np.savez_compressed(
        os.path.join(HERE, "golden_detect.npz"), seed_kwargs=repr(SEED), st=st, tF=tF,
        iC=ops["iC"].numpy(), iC2=ops["iC2"].numpy(), weigh=ops["weigh"].numpy(),
        ycup=ops["ycup"], xcup=ops["xcup"], wTEMP=w["wTEMP"], wPCA=w["wPCA"],
        dmin=np.float64(ops["dmin"]))
    print(f"detect: {len(st)} spikes, {ops['iC'].shape[1]} template positions")
