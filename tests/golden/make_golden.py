"""Generate golden vectors by running the reference's own template matching.

Run from the repository root in a container that has the reference checkout:

    python tests/golden/make_golden.py path/to/reference

The reference package cannot be imported whole offline (its ``__init__``
pulls in faiss and matplotlib), so a namespace stub is registered for
``kilosort`` and only ``kilosort.template_matching`` (plus its light imports
``CCG`` and ``utils``) is loaded from the checkout.  Each case runs the
reference's `prepare_matching`, `run_matching`, `prepare_extract` and
`extract` on CPU tensors drawn by ``kilosort_b200.synth`` and stores inputs
(or their SHA-256 when they are regenerated from the seed) and outputs in
``tests/golden/*.npz``.
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
    from kilosort import template_matching
    return template_matching


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# name -> (make_recording kwargs, Th_learned, max_peels, store_inputs)
CASES = {
    "tiny": (dict(seed=11, n_chan=16, probe="linear", n_templates=12,
                  batch_lengths=[1500]), 8.0, 100, True),
    "small": (dict(seed=12, n_chan=32, probe="np1", n_templates=24,
                   batch_lengths=[4000], rate_hz=(10.0, 30.0)), 8.0, 100, False),
    "nt41": (dict(seed=13, n_chan=24, probe="linear", n_templates=16,
                  batch_lengths=[3000], nt=41, n_pcs=4, t_trough=13,
                  rate_hz=(10.0, 30.0)), 7.0, 100, False),
    "maxpeels2": (dict(seed=12, n_chan=32, probe="np1", n_templates=24,
                       batch_lengths=[4000], rate_hz=(10.0, 30.0)), 8.0, 2, False),
    "empty": (dict(seed=14, n_chan=16, probe="linear", n_templates=8,
                   batch_lengths=[2000]), 1000.0, 100, False),
    "dups": (dict(seed=15, n_chan=32, probe="np1", n_templates=24,
                  batch_lengths=[4000], rate_hz=(10.0, 30.0),
                  duplicate_pairs=3), 8.0, 100, False),
    "cfg1": (dict(seed=1001, n_chan=96, probe="linear", n_templates=80,
                  batch_lengths=[60000], rate_hz=(5.0, 5.0),
                  amp_sd=(8.0, 25.0)), 8.0, 100, False),
}


def run_case(tm, name, kw, Th, max_peels, store_inputs):
    rec = synth.make_recording(**kw)
    nt = rec.nt
    X = torch.from_numpy(np.ascontiguousarray(rec.batch(0)))
    U = torch.from_numpy(rec.U)
    W = torch.from_numpy(rec.wPCA)
    ops = dict(Th_learned=Th, nt=nt, max_peels=max_peels, wPCA=W)
    ctc = tm.prepare_matching(ops, U)
    st, amps, th_amps, Xres = tm.run_matching(ops, X.clone(), U, ctc,
                                              device=torch.device("cpu"))
    Xn, Xr = X.numpy(), Xres.numpy()
    changed = np.flatnonzero(Xn.ravel() != Xr.ravel())
    out = dict(
        seed_kwargs=np.array(repr(kw)), Th=np.float64(Th),
        max_peels=np.int64(max_peels), nt=np.int64(nt),
        X_sha=np.array(sha(Xn)), U_sha=np.array(sha(rec.U)),
        W_sha=np.array(sha(rec.wPCA)), ctc_sha=np.array(sha(ctc.numpy())),
        st=st.numpy(), amps=amps.numpy(), th_amps=th_amps.numpy(),
        xres_sha=np.array(sha(Xr)),
        xres_sum=np.float64(Xr.astype(np.float64).sum()),
        xres_sumsq=np.float64((Xr.astype(np.float64) ** 2).sum()),
    )
    if changed.size <= 400000:
        out["xres_idx"] = changed.astype(np.int64)
        out["xres_val"] = Xr.ravel()[changed]
    if store_inputs:
        out.update(X=Xn, U=rec.U, W=rec.wPCA, ctc=ctc.numpy())
    if name == "small":
        iCC, mask, iU, Ucc = tm.prepare_extract(rec.xc, rec.yc, U, 10, 100,
                                                device=torch.device("cpu"))
        out.update(xc=rec.xc, yc=rec.yc, iCC=iCC.numpy(), iCC_mask=mask.numpy(),
                   iU=iU.numpy(), Ucc=Ucc.numpy(), ctc_full=ctc.numpy())
    print(f"{name}: C={rec.n_chan} K={rec.n_templates} L={X.shape[1]} "
          f"spikes={len(st)} changed={changed.size}")
    np.savez_compressed(os.path.join(HERE, f"golden_{name}.npz"), **out)


def run_extract(tm):
    """Reference `extract` over three equal batches with a synthetic source."""
    kw = dict(seed=21, n_chan=32, probe="np1", n_templates=24,
              batch_lengths=[3000, 3000, 3000], rate_hz=(10.0, 30.0))
    rec = synth.make_recording(**kw)
    bfile = synth.SyntheticBinary(rec, device="cpu")
    W = torch.from_numpy(rec.wPCA)
    ops = dict(Th_learned=8.0, nt=61, max_peels=100, wPCA=W, nt0min=20,
               batch_size=3000, xc=rec.xc, yc=rec.yc,
               settings=dict(nearest_chans=10, position_limit=100, n_pcs=6))
    U = torch.from_numpy(rec.U)
    st, tF, ops = tm.extract(ops, bfile, U, device=torch.device("cpu"))
    print(f"extract: spikes={len(st)}")
    np.savez_compressed(os.path.join(HERE, "golden_extract.npz"),
                        seed_kwargs=np.array(repr(kw)),
                        signal_sha=np.array(sha(rec.signal)),
                        U_sha=np.array(sha(rec.U)), st=st, tF=tF.numpy(),
                        iCC=ops["iCC"].numpy(), iU=ops["iU"].numpy())


if __name__ == "__main__":
    ref = reference_path()
    torch.set_num_threads(max(1, os.cpu_count() or 1))
    tm = load_reference(ref)
    for name, (kw, Th, mp, store) in CASES.items():
        run_case(tm, name, kw, Th, mp, store)
    run_extract(tm)
