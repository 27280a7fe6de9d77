"""Spike-set comparison used by the parity tests and the benchmark."""
import numpy as np


def agreement(st_a, st_r, amps_a=None, amps_r=None):
    """Exact (time, template) agreement between two spike lists.

    Returns dict(matched, n_a, n_r, agreement = min(m/n_r, m/n_a),
    amp_rel_max, amp_rel_p999) where amplitude errors are over matched pairs
    (first unmatched occurrence pairs with first, for duplicates).
    """
    a = np.asarray(st_a)[:, :2].astype(np.int64)
    r = np.asarray(st_r)[:, :2].astype(np.int64)
    key_a = a[:, 0] * 1_000_003 + a[:, 1]
    key_r = r[:, 0] * 1_000_003 + r[:, 1]
    oa = np.argsort(key_a, kind="stable")
    orr = np.argsort(key_r, kind="stable")
    ka, kr = key_a[oa], key_r[orr]
    i = j = 0
    pairs = []
    while i < len(ka) and j < len(kr):
        if ka[i] == kr[j]:
            pairs.append((oa[i], orr[j]))
            i += 1
            j += 1
        elif ka[i] < kr[j]:
            i += 1
        else:
            j += 1
    m = len(pairs)
    na, nr = len(a), len(r)
    if na == 0 and nr == 0:
        agr = 1.0
    elif na == 0 or nr == 0:
        agr = 0.0
    else:
        agr = min(m / nr, m / na)
    out = dict(matched=m, n_a=na, n_r=nr, agreement=agr, amp_rel_max=0.0,
               amp_rel_p999=0.0)
    if amps_a is not None and m:
        pa = np.array([p[0] for p in pairs])
        pr = np.array([p[1] for p in pairs])
        va = np.asarray(amps_a).reshape(-1)[pa].astype(np.float64)
        vr = np.asarray(amps_r).reshape(-1)[pr].astype(np.float64)
        rel = np.abs(va - vr) / np.maximum(np.abs(vr), 1e-30)
        out["amp_rel_max"] = float(rel.max())
        out["amp_rel_p999"] = float(np.quantile(rel, 0.999))
    return out
