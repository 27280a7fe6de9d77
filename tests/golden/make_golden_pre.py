"""Golden vectors of the reference's batch preprocessing.

Run from the repository root in a container that has the reference checkout:

    python tests/golden/make_golden_pre.py path/to/reference

Builds seeded raw int16 batches (kilosort_b200.synth.raw_batch), padded as a
batch is, and runs the reference's own ``BinaryFiltered.filter``
(kilosort/io.py:994-1026) on them, with its high-pass filter
(preprocessing.get_highpass_filter, :121-136) and, for the drift case, its
drift matrix (preprocessing.get_drift_matrix, :44-69, with iKxx formed as
datashift.py:216-223).  ``filter`` only reads the object's settings, so it is
called on a plain namespace.  ``faiss`` (imported by clustering_qr, which
io.py reaches) is replaced by an empty module.  Writes
tests/golden/golden_pre.npz: per case the settings, the whitening matrix and
the reference's output; the inputs are regenerated from their seeds (their
hashes are stored).
"""
import hashlib
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from kilosort_b200 import synth  # noqa: E402

N_CHAN_BIN = 16
CHAN_MAP = np.array([3, 0, 1, 2, 5, 4, 7, 6, 9, 8, 12, 11], dtype=np.int64)
# name: (seed, L, invert_sign, do_CAR, highpass, artifact_threshold, whiten, drift)
CASES = {
    "car": (701, 1100, False, True, True, np.inf, True, None),
    "nocar_invert": (702, 1100, True, False, True, np.inf, True, None),
    "artifact": (703, 1100, False, True, True, 40.0, True, None),
    "drift": (704, 1100, False, True, True, np.inf, True, 7.5),
    "nohp": (705, 1100, False, True, False, np.inf, False, None),
    "odd": (706, 1101, False, True, True, 1e9, True, None),
    "car_invert": (707, 1100, True, True, True, np.inf, True, None),
    "car_invert_nohp": (708, 1100, True, True, False, np.inf, False, None),
}


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
    from kilosort import io as kio, preprocessing as kpre
    return kio, kpre


def whiten_matrix(seed, C):
    rng = np.random.default_rng(seed)
    return (np.eye(C) + 0.15 * rng.standard_normal((C, C))).astype(np.float32)


def probe(C):
    xc = np.tile(np.array([0.0, 20.0], np.float32), C // 2 + 1)[:C]
    yc = (20.0 * (np.arange(C) // 2)).astype(np.float32)
    return xc, yc


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


if __name__ == "__main__":
    ref = reference_path()
    kio, kpre = load_reference(ref)
    cpu = torch.device("cpu")
    hp = kpre.get_highpass_filter(30000, 300, device=cpu)
    C = len(CHAN_MAP)
    out = {"chan_map": CHAN_MAP, "n_chan_bin": N_CHAN_BIN}
    for name, (seed, L, inv, car, use_hp, thr, use_w, shift) in CASES.items():
        raw = synth.raw_batch(seed, N_CHAN_BIN, L)
        W = whiten_matrix(seed, C)
        ops = None
        dshift = None
        if shift is not None:
            xc, yc = probe(C)
            xp = np.vstack((xc, yc)).T
            Kxx = torch.from_numpy(kpre.kernel2D_torch(torch.from_numpy(xp), torch.from_numpy(xp),
                                                       20.0).numpy())
            ops = {"yblk": np.array([0.0]), "nblocks": 1, "probe": {"xc": xc, "yc": yc},
                   "settings": {"sig_interp": 20.0},
                   "iKxx": torch.linalg.inv(Kxx + 0.01 * torch.eye(C))}
            dshift = np.array([[shift]], dtype=np.float32)
            out[f"{name}_xc"], out[f"{name}_yc"] = xc, yc
        self = types.SimpleNamespace(
            chan_map=CHAN_MAP, invert_sign=inv, do_CAR=car, hp_filter=hp if use_hp else None,
            artifact_threshold=thr, whiten_mat=torch.from_numpy(W) if use_w else None,
            dshift=dshift, device=cpu)
        X = torch.from_numpy(raw.T.astype(np.float32))
        Y = kio.BinaryFiltered.filter(self, X, ops, 0 if dshift is not None else None)
        out[f"{name}_out"] = Y.numpy().astype(np.float32)
        out[f"{name}_W"] = W
        out[f"{name}_raw_sha"] = sha(raw)
        out[f"{name}_params"] = np.array([seed, L, inv, car, use_hp, use_w,
                                          -1.0 if shift is None else shift], np.float64)
        out[f"{name}_thr"] = np.float64(thr)
        print(name, Y.shape, float(Y.abs().max()))
    np.savez_compressed(os.path.join(HERE, "golden_pre.npz"), **out)
