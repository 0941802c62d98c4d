"""C ABI checks that need no GPU: the library loads, exports every function
include/iac_b200.h declares, and its host-side geometry and argument checks
behave like the reference's."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from incohautocorrelate_b200 import capi
from helpers import mesh_shape_dict, small_detector

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "iac_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(iac_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(capi.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version_and_status_strings():
    L = capi.lib()
    assert L.iac_abi_version() == 1
    assert L.iac_status_string(0) == b"ok"
    assert b"outside the mesh" in L.iac_status_string(capi.IAC_ERR_OUT_OF_MESH)


@pytest.mark.parametrize("edge,zoom", [(63, 1.0), (199, 1.0), (253, 1.0), (31, 2.0)])
def test_big_mesh_shape_matches_reference_sizing(oracle_lib, edge, zoom):
    for mq in ([0.0951, 0.0951, 0.00453], [0.717, 0.371, 0.07], [0.3, 0.9, 0.2]):
        got = mesh_shape_dict(capi.big_mesh_shape(mq, edge, zoom))
        want = mesh_shape_dict(oracle_lib.big_mesh_shape(mq, edge, zoom))
        assert got == want


@pytest.mark.parametrize("perp,zoom", [(63, 1.0), (253, 1.0), (101, 1.5)])
def test_small_cq_mesh_shape_matches_reference_sizing(oracle_lib, perp, zoom):
    for mq in ([0.717, 0.371, 0.07], [0.2, 0.9, 0.5], [0.05, 0.06, 0.9]):
        got = mesh_shape_dict(capi.small_cq_mesh_shape(mq, perp, zoom))
        want = mesh_shape_dict(oracle_lib.small_cq_mesh_shape(mq, perp, zoom))
        assert got == want


def test_ac1d_shape_matches(oracle_lib):
    mq = [0.717, 0.371, 0.07]
    a = capi.ac1d_shape(mq, 2048, 1.0)
    b = oracle_lib.ac1d_shape(mq, 2048, 1.0)
    assert (a.size, a.max_q, a.dq_per_step) == (b.size, b.max_q, b.dq_per_step)


def test_even_mesh_rejected_with_message():
    with pytest.raises(capi.IacError) as e:
        capi.big_mesh_shape([0.1, 0.1, 0.1], 64)
    assert e.value.status == capi.IAC_ERR_INVALID_ARG
    assert "odd" in str(e.value)


def test_mesh_word_counts():
    assert capi.half_mesh_words(201) == 201 * 201 * 101
    assert capi.full_mesh_words(65) == 65 ** 3


def test_null_context_rejected():
    L = capi.lib()
    p = capi.sparse_params(capi.big_mesh_shape([0.1, 0.1, 0.01], 31))
    st = L.iac_sparse_ac_batch(None, None, None, None, 1, C.byref(p), None, None)
    assert st == capi.IAC_ERR_INVALID_ARG


def test_workload_generators_are_seeded_and_shaped():
    from incohautocorrelate_b200 import workloads as W
    a = W.small_config(nframes=50, seed=1)
    b = W.small_config(nframes=50, seed=1)
    np.testing.assert_array_equal(a["photons"], b["photons"])
    assert a["offsets"][-1] == len(a["photons"])
    n = np.diff(a["offsets"].astype(np.int64))
    assert 100 < n.mean() < 230  # Poisson(0.01) over 16384 pixels
    R = W.haar_rotations(1000, 3).reshape(-1, 3, 3).astype(np.float64)
    np.testing.assert_allclose(R @ R.transpose(0, 2, 1), np.broadcast_to(np.eye(3), R.shape),
                               atol=1e-6)
