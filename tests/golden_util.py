"""Helpers to load golden vectors made by tests/golden/make_golden.py."""
import ast
import hashlib
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["tiny", "small", "nt41", "maxpeels2", "empty", "dups", "cfg1"]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def load(name):
    return dict(np.load(os.path.join(GOLDEN, f"golden_{name}.npz")))


def case_inputs(g):
    """Regenerate (rec, X, U, W) of a golden case and check their hashes."""
    from kilosort_b200 import synth
    kw = ast.literal_eval(str(g["seed_kwargs"]))
    rec = synth.make_recording(**kw)
    X = np.ascontiguousarray(rec.batch(0))
    assert sha(X) == str(g["X_sha"]), "generator no longer reproduces X"
    assert sha(rec.U) == str(g["U_sha"]), "generator no longer reproduces U"
    assert sha(rec.wPCA) == str(g["W_sha"]), "generator no longer reproduces wPCA"
    return rec, X, rec.U, rec.wPCA


def xres_from_golden(g, X):
    """Rebuild the reference residual from the stored changed entries."""
    Xr = X.copy().ravel()
    Xr[g["xres_idx"]] = g["xres_val"]
    return Xr.reshape(X.shape)
