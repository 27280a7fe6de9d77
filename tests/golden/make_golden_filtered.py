"""Golden vectors of the reference's ``extract`` over its own ``BinaryFiltered``.

Run from the repository root in a container that has the reference checkout:

    python tests/golden/make_golden_filtered.py path/to/reference

Builds a seeded raw int16 file (kilosort_b200.synth.raw_recording: 64
recording channels on a permutation of 66 file channels, a ragged last
batch), wraps it in the reference's own ``io.BinaryFiltered``
(kilosort/io.py:968-1045, ``file_object`` = the array, NT = 3000) with the
reference's high-pass filter (preprocessing.get_highpass_filter), a whitening
matrix, and per-batch drift over two blocks (``iKxx`` formed as
datashift.py:216-223), then runs the reference's ``template_matching.extract``
on CPU.  Writes tests/golden/golden_filtered.npz: the settings, the
reference's batch count and edges, a hash of each padded raw window
(``BinaryRWFile.padded_batch_to_torch``, io.py:789-831, before the filter),
the drift matrices of the first and last batch, 16 rows of the filtered last
batch, and extract's ``st``, ``tF``, ``iCC``, ``iU``.  The raw file is
regenerated from its seeds (its hash is stored).
"""
import hashlib
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from kilosort_b200 import synth  # noqa: E402
import make_golden_pre as mkpre  # noqa: E402

REC = dict(seed=9201, n_chan=64, probe="np1", n_templates=40,
           batch_lengths=[3000] * 5 + [1000], rate_hz=(10.0, 30.0))
RAW_SEED = 9202
N_CHAN_BIN = 66
NT, NT_WAVE = 3000, 61
GAIN = 25.0
SIG_INTERP = 20.0
N_ROWS_SAVED = 16


def chan_map():
    """Recording channel c lives on file channel chan_map[c] (two file
    channels carry nothing)."""
    return np.random.default_rng(9203).permutation(N_CHAN_BIN)[:REC["n_chan"]].astype(np.int64)


def whitening(C):
    rng = np.random.default_rng(9204)
    return ((np.eye(C) + 0.03 * rng.standard_normal((C, C))) / GAIN).astype(np.float32)


def drift_setup(rec, n_batches):
    """(ops entries of the drift correction, dshift [n_batches, 3])."""
    rng = np.random.default_rng(9205)
    yc = rec.yc.astype(np.float32)
    yblk = np.array([yc.min() + 0.25 * np.ptp(yc), yc.mean(), yc.max() - 0.25 * np.ptp(yc)])
    dshift = rng.uniform(-6.0, 6.0, (n_batches, 3))
    return yblk, dshift


def make_raw(rec):
    return synth.raw_recording(rec, N_CHAN_BIN, chan_map(), RAW_SEED, gain=GAIN)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


if __name__ == "__main__":
    kio, kpre = mkpre.load_reference(mkpre.reference_path())
    from kilosort import datashift, template_matching as tm
    cpu = torch.device("cpu")
    rec = synth.make_recording(**REC)
    raw = make_raw(rec)
    C = rec.n_chan
    xc, yc = rec.xc.astype(np.float32), rec.yc.astype(np.float32)
    hp = kpre.get_highpass_filter(30000, 300, device=cpu)
    W = torch.from_numpy(whitening(C))
    n_guess = int(np.ceil(raw.shape[0] / NT))
    yblk, dshift = drift_setup(rec, n_guess)
    bfile = kio.BinaryFiltered(None, N_CHAN_BIN, 30000, NT, NT_WAVE, 20, chan_map(),
                               hp_filter=hp, whiten_mat=W, dshift=dshift, device=cpu,
                               file_object=raw)
    nb = int(bfile.n_batches)
    xp = np.vstack((xc, yc)).T
    Kxx = torch.from_numpy(datashift.kernel2D(xp, xp, SIG_INTERP))
    iKxx = torch.linalg.inv(Kxx + 0.01 * torch.eye(Kxx.shape[0]))
    ops = dict(Th_learned=8.0, nt=NT_WAVE, max_peels=100, wPCA=torch.from_numpy(rec.wPCA),
               nt0min=20, batch_size=NT, xc=xc, yc=yc, nblocks=2, yblk=yblk,
               probe=dict(xc=xc, yc=yc), iKxx=iKxx,
               settings=dict(nearest_chans=10, position_limit=100, n_pcs=6,
                             sig_interp=SIG_INTERP))
    edges = np.array([bfile._get_batch_edges(b) for b in range(nb)], np.int64)
    windows = []
    for b in range(nb):
        X = kio.BinaryRWFile.padded_batch_to_torch(bfile, b)
        assert torch.equal(X, X.round())
        windows.append(sha(X.numpy().astype(np.int16)))
    M0 = kpre.get_drift_matrix(ops, dshift[0], device=cpu)
    Mlast = kpre.get_drift_matrix(ops, dshift[nb - 1], device=cpu)
    Xlast = bfile.padded_batch_to_torch(nb - 1, ops)
    st, tF, ops_out = tm.extract(ops, bfile, torch.from_numpy(rec.U), device=cpu)
    np.savez_compressed(
        os.path.join(HERE, "golden_filtered.npz"), rec_kwargs=repr(REC), raw_sha=sha(raw),
        n_chan_bin=N_CHAN_BIN, NT=NT, chan_map=chan_map(), W=W.numpy(), dshift=dshift,
        yblk=yblk, xc=xc, yc=yc, iKxx=iKxx.numpy(), sig_interp=SIG_INTERP,
        n_batches=nb, imax=int(bfile.imax), edges=edges, window_sha=np.array(windows),
        M0=M0.numpy(), Mlast=Mlast.numpy(), Xlast_rows=Xlast[:N_ROWS_SAVED].numpy(),
        st=st, tF=tF.numpy(), iCC=ops_out["iCC"].numpy(), iU=ops_out["iU"].numpy())
    print(f"filtered extract: {nb} batches, {len(st)} spikes, raw {raw.shape}")
