"""Batch cutting of the streaming matcher (host logic, no GPU): the padded
windows equal those kilosort/io.py builds (first batch's left pad repeats its
first sample and, when it is the only batch, zeros follow its data; a later
batch that ends early is padded with its last sample)."""
import numpy as np
import pytest

from kilosort_b200.stream import batch_windows, padded_raw_window


def _io_window(raw, b, NT, nt):
    """Literal restatement of io.py:771-831 (edges of batch b, padding)."""
    n = raw.shape[0]
    n_batches = int(np.ceil(n / NT))
    if b == 0:
        bstart, bend = 0, NT + nt
    else:
        bstart = b * NT - nt
        bend = min(n, bstart + NT + 2 * nt)
    data = raw[bstart:bend].T
    X = np.zeros((raw.shape[1], NT + 2 * nt), raw.dtype)
    nsamp = data.shape[-1]
    if b == 0:
        X[:, nt:nt + nsamp] = data
        X[:, :nt] = X[:, nt:nt + 1]
    elif b == n_batches - 1:
        X[:, :nsamp] = data
        X[:, nsamp:] = X[:, nsamp - 1:nsamp]
    else:
        X[:] = data
    return X.T


@pytest.mark.parametrize("n", [9000, 9500, 2999, 12122])
def test_batch_windows_cut_as_io_does(n):
    rng = np.random.default_rng(n)
    raw = rng.integers(-100, 100, size=(n, 5), dtype=np.int16)
    NT, nt = 3000, 61
    nb = len(batch_windows(n, NT, nt))
    assert nb == int(np.ceil(n / NT))
    for b in range(nb):
        out = np.empty((NT + 2 * nt, 5), np.int16)
        np.testing.assert_array_equal(padded_raw_window(raw, b, NT, nt, out), _io_window(raw, b, NT, nt))


