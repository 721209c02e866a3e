"""CPU checks of the C ABI boundary: the library loads, exports every entry
point include/tmnb.h declares, and argument errors surface as RuntimeError
with the reference's messages (no GPU needed for any of these)."""

import ctypes
import os
import re

import numpy as np
import pytest

from timemachine_b200 import _lib
from timemachine_b200 import potentials as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "tmnb.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"\b(tmnb_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_library_version_and_error_string():
    lib = _lib.lib()
    assert b"sm_100a" in lib.tmnb_version()
    assert isinstance(lib.tmnb_last_error(), bytes)


def test_null_handle_is_an_error_not_a_crash():
    lib = _lib.lib()
    rc = lib.tmnb_potential_set_nblist_padding(None, 0.1)
    assert rc == 1
    assert b"null" in lib.tmnb_last_error()
    assert lib.tmnb_potential_destroy(None) == 0
    assert lib.tmnb_potential_num_params(None) == -1


def test_unsupported_precision_rejected():
    lib = _lib.lib()
    plane = np.zeros(4, np.int32)
    h = ctypes.c_void_p()
    rc = lib.tmnb_all_pairs_create(
        4, plane.ctypes.data_as(ctypes.c_void_p), plane.ctypes.data_as(ctypes.c_void_p), 2.0, 1.2, None, 0, 0, 64,
        ctypes.byref(h),
    )
    assert rc == 5  # TMNB_ERR_UNSUPPORTED
    with pytest.raises(RuntimeError, match="float32"):
        P.NonbondedAllPairs(plane, plane, 2.0, 1.2).unbound_impl(np.float64)


def test_all_pairs_argument_errors():
    """tests/nonbonded/test_nonbonded_all_pairs.py:14-26."""
    with pytest.raises(RuntimeError, match="lambda offset idxs and plane idxs need to be equivalent"):
        P.NonbondedAllPairs([0], [0, 0], 2.0, 1.1).unbound_impl(np.float32)
    with pytest.raises(RuntimeError, match="atom indices must be unique"):
        P.NonbondedAllPairs([0, 1], [0, 0], 2.0, 1.1, [0, 0]).unbound_impl(np.float32)


def test_pair_list_argument_errors():
    """tests/nonbonded/test_nonbonded_pair_list.py:18-32 (the size checks need no GPU)."""
    with pytest.raises(RuntimeError, match="pair_idxs.size\\(\\) must be even, but got 1"):
        P.NonbondedPairList([0], [0], [0], [0], 2.0, 1.1).unbound_impl(np.float32)
    with pytest.raises(RuntimeError, match="expected same number of pairs and scale tuples, but got 1 != 2"):
        P.NonbondedPairList([(0, 1)], [(1, 1), (2, 2)], [0, 0], [0, 0], 2.0, 1.1).unbound_impl(np.float32)


def test_nonbonded_rejects_duplicate_exclusions():
    """timemachine/lib/potentials.py:270-280."""
    with pytest.raises(AssertionError):
        P.Nonbonded(np.array([[0, 1], [1, 0]]), np.ones((2, 2)), [0, 0], [0, 0], 2.0, 1.2)


def test_create_without_gpu_fails_loudly():
    """On a machine without a CUDA device, creation reports a CUDA error (no CPU fallback)."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError):
        P.NonbondedAllPairs(np.zeros(8, np.int32), np.zeros(8, np.int32), 2.0, 1.2).unbound_impl(np.float32)


def test_bound_impl_requires_params():
    with pytest.raises(ValueError, match="not been bound"):
        P.NonbondedAllPairs([0], [0], 2.0, 1.1).bound_impl(np.float32)
