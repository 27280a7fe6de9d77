"""C-ABI library checks that need no GPU: it loads, exports every declared
symbol, and its host-side queries answer."""
import ctypes

import pytest

from kilosort_b200 import _lib


def test_library_loads_and_exports_header_symbols():
    lib = _lib.load()
    declared = _lib.header_symbols()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in include/ks_b200.h but not exported"
    # every binding we set up corresponds to a declared function
    assert set(_lib.SIGNATURES) == set(declared)


def test_status_strings_and_version():
    lib = _lib.load()
    assert lib.ks_version() >= 1
    assert lib.ks_status_string(0) == b"ok"
    assert b"overflow" in lib.ks_status_string(_lib.KS_ERR_OVERFLOW)
    assert b"timed out" in lib.ks_status_string(_lib.KS_ERR_TIMEOUT)


def test_workspace_queries():
    lib = _lib.load()
    C, L, K, P = 384, 60122, 600, 6
    fp32 = lib.ks_project_workspace_size(C, L, K, P, _lib.KS_PROJ_FP32)
    split = lib.ks_project_workspace_size(C, L, K, P, _lib.KS_PROJ_BF16X3)
    # Yt: Lpad * Q floats (fp32) vs two bf16 planes -> same size; both > Y bytes
    assert fp32 >= 60160 * 2304 * 4
    assert split >= 60160 * 2304 * 4
    peel = lib.ks_peel_workspace_size(L, K, 61, _lib.KS_B_ROWS, _lib.KS_CTC_KJL)
    assert peel >= K * L * 4                     # tiled copy of a row-major B
    assert lib.ks_peel_workspace_size(L, K, 61, _lib.KS_B_TILED, _lib.KS_CTC_KJL) < K * L
    # the reference ctc layout adds room for its transposed copy
    assert lib.ks_peel_workspace_size(L, K, 61, _lib.KS_B_ROWS, _lib.KS_CTC_JKL) >= \
        peel + K * K * 123 * 4
    total = lib.ks_run_matching_workspace_size(C, L, K, P, 61, _lib.KS_PROJ_FP32,
                                               _lib.KS_CTC_KJL)
    assert total >= fp32 + K * L * 4
    assert lib.ks_ctc_workspace_size(K, P, C, 61) >= (K * P) ** 2 * 4


def test_peel_rejects_bad_arguments_before_touching_the_device():
    lib = _lib.load()
    # null pointers -> KS_ERR_ARG
    rc = lib.ks_peel(None, 64, _lib.KS_B_ROWS, None, None, None, None, _lib.KS_CTC_JKL, None,
                     4, 64, 2, 6, 61, 64.0, 100, 10, None, None, None, None, None, 0, None)
    assert rc == _lib.KS_ERR_ARG
    assert b"null" in lib.ks_last_error()


def test_python_layer_refuses_cpu_tensors():
    import torch
    import kilosort_b200 as kb
    ops = dict(Th_learned=8.0, nt=61, max_peels=100, wPCA=torch.zeros(6, 61))
    with pytest.raises(ValueError, match="CUDA"):
        kb.run_matching(ops, torch.zeros(4, 200), torch.zeros(2, 6, 4),
                        torch.zeros(2, 2, 123))


def test_descriptor_structs_match_the_c_layout(tmp_path):
    """ks_rec_desc / ks_batch_desc: ctypes mirrors agree with the C compiler."""
    import os
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "ks_b200.h"\n'
        "int main(void) {\n"
        '  printf("%zu %zu %zu %zu %zu\\n", sizeof(ks_rec_desc), offsetof(ks_rec_desc, th2),\n'
        "         offsetof(ks_rec_desc, max_peels), offsetof(ks_rec_desc, capacity),\n"
        "         offsetof(ks_rec_desc, nt));\n"
        '  printf("%zu %zu %zu %zu\\n", sizeof(ks_batch_desc), offsetof(ks_batch_desc, L),\n'
        "         offsetof(ks_batch_desc, rec), offsetof(ks_batch_desc, info));\n"
        "  return 0;\n}\n")
    exe = tmp_path / "layout"
    inc = os.path.join(os.path.dirname(_lib.HEADER))
    subprocess.run([cc, "-I", inc, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    r = [int(v) for v in out[0].split()]
    b = [int(v) for v in out[1].split()]
    R, B = _lib.RecDesc, _lib.BatchDesc
    assert r == [ctypes.sizeof(R), R.th2.offset, R.max_peels.offset, R.capacity.offset,
                 R.nt.offset]
    assert b == [ctypes.sizeof(B), B.L.offset, B.rec.offset, B.info.offset]


def test_batched_workspace_query_and_argument_checks():
    lib = _lib.load()
    recs = (_lib.RecDesc * 2)(
        _lib.RecDesc(1, 1, 1, 384, 600, 6, 61, 64.0, 100, 100000),
        _lib.RecDesc(1, 1, 1, 96, 150, 6, 61, 64.0, 100, 100000))
    bats = (_lib.BatchDesc * 3)(
        _lib.BatchDesc(1, 1, 60122, 0, 1, 1, 1, 1),
        _lib.BatchDesc(1, 1, 20122, 1, 1, 1, 1, 1),
        _lib.BatchDesc(1, 1, 8122, 0, 1, 1, 1, 1))
    n_split = lib.ks_match_batches_workspace_size(recs, 2, bats, 3, _lib.KS_PROJ_BF16X3, 2)
    n_fp32 = lib.ks_match_batches_workspace_size(recs, 2, bats, 3, _lib.KS_PROJ_FP32, 2)
    # tiled scores of every batch at least
    assert n_split > 4 * (600 * 60122 + 150 * 20122 + 600 * 8122)
    assert n_fp32 > 4 * (600 * 60122 + 150 * 20122 + 600 * 8122)
    # split form stacks the bf16 hi/lo projections of every batch of a recording
    assert n_split > 2 * 2 * (60160 + 8192) * 2304
    # more teams, more team scratch
    assert lib.ks_match_batches_workspace_size(recs, 2, bats, 3, _lib.KS_PROJ_BF16X3, 3) > n_split
    # a bad recording index, too many batches and a bad precision are refused
    bats[1].rec = 5
    assert lib.ks_match_batches_workspace_size(recs, 2, bats, 3, _lib.KS_PROJ_BF16X3, 2) == 0
    assert b"recording index" in lib.ks_last_error()
    bats[1].rec = 1
    assert lib.ks_match_batches_workspace_size(recs, 2, bats, 300, _lib.KS_PROJ_BF16X3, 2) == 0
    assert lib.ks_match_batches_workspace_size(recs, 2, bats, 3, 7, 2) == 0
    rc = lib.ks_match_batches(recs, 2, bats, 3, _lib.KS_PROJ_BF16X3, 2, 1, None, 0, None, None)
    assert rc == _lib.KS_ERR_WORKSPACE


def test_static_peel_limits_are_checked_before_the_device():
    """ks_peel_static refuses, with a message, a batch longer than its fixed
    array holds and, at that longest batch, more templates than the array
    holds; both checks come before any device call."""
    lib = _lib.load()
    max_l, max_k = 131072, 56896
    rc = lib.ks_peel_static(None, None, None, None, None, None, 4, max_l + 1, 2, 6, 61, 64.0,
                            1, 1, None, None, None, None, None)
    assert rc == _lib.KS_ERR_UNSUPPORTED
    assert b"131072" in lib.ks_last_error()
    rc = lib.ks_peel_static(None, None, None, None, None, None, 4, max_l, max_k + 1, 6, 61,
                            64.0, 1, 1, None, None, None, None, None)
    assert rc == _lib.KS_ERR_UNSUPPORTED
    msg = lib.ks_last_error()
    assert b"K=56897" in msg and b"56896" in msg
