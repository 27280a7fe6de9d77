"""ctypes binding of ``libks_b200.so`` (the C ABI in ``include/ks_b200.h``).

The library is built in-tree by ``python -m kilosort_b200.build``.  Loading it
needs no GPU (the CUDA runtime is linked statically); calling any compute entry
point needs a B200.  There is no fallback: if the library is missing, every
compute call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libks_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "ks_b200.h")

KS_OK = 0
KS_ERR_ARG = 1
KS_ERR_CUDA = 2
KS_ERR_OVERFLOW = 3
KS_ERR_TIMEOUT = 4
KS_ERR_WORKSPACE = 5
KS_ERR_UNSUPPORTED = 6
KS_ERR_DEGENERATE = 7

KS_PROJ_FP32 = 0
KS_PROJ_BF16X3 = 1

KS_CTC_JKL = 0
KS_CTC_KJL = 1

KS_B_ROWS = 0
KS_B_TILED = 1

_i64, _f32, _int, _sz, _vp = C.c_int64, C.c_float, C.c_int, C.c_size_t, C.c_void_p

# name -> (restype, argtypes); pointers are passed as integers (c_void_p)
SIGNATURES = {
    "ks_version": (_int, []),
    "ks_status_string": (C.c_char_p, [_int]),
    "ks_last_error": (C.c_char_p, []),
    "ks_template_energy": (_int, [_vp, _i64, _i64, _i64, _vp, _vp]),
    "ks_project_workspace_size": (_sz, [_i64, _i64, _i64, _i64, _int]),
    "ks_project": (_int, [_vp, _vp, _vp, _i64, _i64, _i64, _i64, _i64, _int, _vp,
                          _i64, _int, _vp, _vp, _sz, _vp]),
    "ks_peel_workspace_size": (_sz, [_i64, _i64, _i64, _int, _int]),
    "ks_peel": (_int, [_vp, _i64, _int, _vp, _vp, _vp, _vp, _int, _vp, _i64, _i64, _i64, _i64,
                       _i64, _f32, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _sz, _vp]),
    "ks_run_matching_workspace_size": (_sz, [_i64, _i64, _i64, _i64, _i64, _int, _int]),
    "ks_run_matching": (_int, [_vp, _vp, _vp, _vp, _int, _i64, _i64, _i64, _i64, _i64,
                               _f32, _i64, _int, _i64, _vp, _vp, _vp, _vp, _vp,
                               _vp, _sz, _vp]),
    "ks_ctc_transpose": (_int, [_vp, _i64, _i64, _vp, _vp]),
    "ks_features": (_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _i64,
                           _i64, _i64, _i64, _i64, _vp, _vp]),
    "ks_features_counted": (_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _i64,
                                   _i64, _i64, _i64, _vp, _i64, _vp, _vp]),
    "ks_template_channels": (_int, [_vp, _vp, _i64, _i64, _i64, _i64, _vp, _vp, _vp]),
    "ks_ctc_workspace_size": (_sz, [_i64, _i64, _i64, _i64]),
    "ks_ctc": (_int, [_vp, _vp, _i64, _i64, _i64, _i64, _vp, _vp, _sz, _vp]),
    "ks_selftest_wait": (_int, [_i64, _vp, _vp]),
    "ks_peel_static": (_int, [_vp, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _i64, _i64, _i64,
                              _f32, _i64, _i64, _vp, _vp, _vp, _vp, _vp]),
    "ks_recon_workspace_size": (_sz, [_i64, _i64, _i64, _i64, _i64, _i64]),
    "ks_recon_loss": (_int, [_vp, _vp, _vp, _i64, _vp, _vp, _i64, _i64, _i64, _i64, _i64,
                             _vp, _vp, _vp, _vp, _sz, _vp]),
    "ks_recon_adjoint": (_int, [_vp, _vp, _vp, _i64, _vp, _vp, _i64, _i64, _i64, _i64, _i64,
                                _vp, _vp, _vp, _vp, _vp, _vp, _sz, _vp]),
    "ks_spike_positions": (_int, [_vp] * 7 + [_i64] * 5 + [_vp] * 5),
    "ks_detect_workspace_size": (_sz, [_i64, _i64, _i64, _i64]),
    "ks_detect": (_int, [_vp, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _vp, _i64, _vp, _i64,
                         _i64, _i64, _f32, _vp, _i64, _vp, _i64, _vp, _vp, _vp, _vp, _vp,
                         _vp, _vp, _vp, _sz, _vp]),
    "ks_similarity_workspace_size": (_sz, [_i64, _i64, _i64, _i64]),
    "ks_similarity": (_int, [_vp, _vp, _i64, _i64, _i64, _i64, _vp, _vp, _sz, _vp]),
    "ks_preprocess_workspace_size": (_sz, [_i64, _i64, _int]),
    "ks_preprocess_int16": (_int, [_vp, _i64, _i64, _vp, _i64, _int, _int, _vp, _i64, _i64,
                                   _f32, _vp, _vp, _i64, _vp, _vp, _sz, _vp]),
    "ks_whiten_int16_workspace_size": (_sz, [_i64, _i64]),
    "ks_whiten_int16": (_int, [_vp, _i64, _i64, _i64, _vp, _f32, _vp, _i64, _vp, _vp, _sz,
                               _vp]),
    "ks_trace_stages": (_int, [_int]),
    "ks_trace_read": (_int, [_vp, _int]),
    "ks_match_batches_workspace_size": (_sz, [_vp, _i64, _vp, _i64, _int, _i64]),
    "ks_match_batches": (_int, [_vp, _i64, _vp, _i64, _int, _i64, _i64, _vp, _sz, _vp, _vp]),
    "ks_remove_duplicates_workspace_size": (_sz, [_i64]),
    "ks_remove_duplicates": (_int, [_vp, _vp, _i64, _i64, _vp, _vp, _sz, _vp]),
    "ks_phy_templates": (_int, [_vp, _vp, _i64, _i64, _i64, _i64, _vp, _vp]),
    "ks_snippets_workspace_size": (_sz, [_i64, _i64]),
    "ks_snippets": (_int, [_vp, _i64, _i64, _i64, _i64, _f32, _i64, _i64, _vp, _vp, _vp, _sz,
                           _vp]),
    "ks_snippet_gram_workspace_size": (_sz, [_i64, _i64]),
    "ks_snippet_gram": (_int, [_vp, _i64, _i64, _vp, _vp, _sz, _vp]),
    "ks_kmeans_workspace_size": (_sz, [_i64, _i64, _i64]),
    "ks_kmeans_step": (_int, [_vp, _i64, _i64, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _sz, _vp]),
    "ks_kmeans_mindist": (_int, [_vp, _i64, _i64, _vp, _int, _vp, _vp]),
    "ks_kmeans_candidates": (_int, [_vp, _i64, _i64, _vp, _i64, _vp, _vp, _vp, _sz, _vp]),
}

KS_MAX_BATCHES = 256
KS_MAX_RECORDINGS = 8


class RecDesc(C.Structure):
    """``ks_rec_desc``: one recording's template set and peel settings."""
    _fields_ = [("U", _vp), ("W", _vp), ("ctcT", _vp), ("C", _i64), ("K", _i64),
                ("P", _i64), ("nt", _i64), ("th2", _f32), ("max_peels", _i64),
                ("capacity", _i64)]


class BatchDesc(C.Structure):
    """``ks_batch_desc``: one padded batch, its recording and its outputs."""
    _fields_ = [("X", _vp), ("Xres", _vp), ("L", _i64), ("rec", _i64), ("st", _vp),
                ("amps", _vp), ("th_amps", _vp), ("info", _vp)]

_lib = None


class KilosortB200Error(RuntimeError):
    """A C-ABI call returned a nonzero status."""

    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


def header_symbols():
    """Names of the functions declared in include/ks_b200.h."""
    with open(HEADER) as f:
        text = f.read()
    return sorted(set(re.findall(r"KS_API\s+[\w\s\*]+?\b(ks_\w+)\s*\(", text)))


def load():
    """Load the shared library once; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m kilosort_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status, what):
    if status != KS_OK:
        lib = load()
        msg = lib.ks_last_error().decode(errors="replace")
        name = lib.ks_status_string(status).decode()
        raise KilosortB200Error(status, f"{what}: {name} ({status}): {msg}")


def status_message(status):
    return load().ks_status_string(int(status)).decode()
