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
    """precision 32 (the _f32 kernels) and 64 (_f64) are built; anything else is refused."""
    lib = _lib.lib()
    plane = np.zeros(4, np.int32)
    h = ctypes.c_void_p()
    rc = lib.tmnb_all_pairs_create(
        4, plane.ctypes.data_as(ctypes.c_void_p), plane.ctypes.data_as(ctypes.c_void_p), 2.0, 1.2, None, 0, 0, 16,
        ctypes.byref(h),
    )
    assert rc == 5  # TMNB_ERR_UNSUPPORTED
    assert b"precision" in lib.tmnb_last_error()
    with pytest.raises(RuntimeError, match="unsupported precision"):
        P.NonbondedAllPairs(plane, plane, 2.0, 1.2).unbound_impl(np.float16)
    with pytest.raises(RuntimeError, match="FP32 arithmetic only"):
        P.HarmonicBond(np.zeros((1, 2), np.int32)).unbound_impl(np.float64)


# The reference test of the four transform expressions
# (tests/test_parameter_interpolation.py:91-140) and their closed forms.
TRANSFORMS = [
    ("lambda", lambda l: l, lambda l: 1.0),
    ("lambda*lambda", lambda l: l * l, lambda l: 2 * l),
    ("sin(lambda*PI/2)", lambda l: np.sin(l * np.pi / 2), lambda l: np.pi / 2 * np.cos(l * np.pi / 2)),
    (
        "lambda < 0.5 ? sin(lambda*PI)*sin(lambda*PI) : 1",
        lambda l: np.sin(l * np.pi) ** 2 if l < 0.5 else 1.0,
        lambda l: 2 * np.pi * np.sin(l * np.pi) * np.cos(l * np.pi) if l < 0.5 else 0.0,
    ),
    ("1-lambda*lambda", lambda l: 1 - l * l, lambda l: -2 * l),
    ("exp(-2.5*lambda) + pow(lambda, 3)", lambda l: np.exp(-2.5 * l) + l**3, lambda l: -2.5 * np.exp(-2.5 * l) + 3 * l**2),
    ("fmax(lambda, 0.25) * (1.0f - tanh(lambda))", None, None),
]


@pytest.mark.parametrize("expr,f,df", TRANSFORMS)
def test_lambda_transform_values_and_derivatives(expr, f, df):
    """Host evaluation of the transform expressions: values against closed
    forms (or numpy), derivatives against closed forms and central differences."""
    for lam in [0.0, 0.2, 0.37, 0.6, 0.7, 0.8, 1.0]:
        v, d = P.lambda_transform(expr, lam)
        if f is not None:
            assert v == pytest.approx(f(lam), rel=1e-14, abs=1e-15)
            assert d == pytest.approx(df(lam), rel=1e-12, abs=1e-13)
        h = 1e-6
        if abs(lam - 0.5) > 2 * h and abs(lam - 0.25) > 2 * h:  # away from the branch points
            fd = (P.lambda_transform(expr, lam + h)[0] - P.lambda_transform(expr, lam - h)[0]) / (2 * h)
            assert d == pytest.approx(fd, rel=1e-6, abs=1e-8)
    # the identity is exact: f = lambda, df = 1, as the reference's complex step gives
    assert P.lambda_transform("lambda", 0.123456789) == (0.123456789, 1.0)


def test_lambda_transform_c_semantics():
    """C rules of the reference's compiled expressions: int / int truncates, float literals round."""
    assert P.lambda_transform("1/2*lambda", 0.8) == (0.0, 0.0)
    assert P.lambda_transform("1.0/2*lambda", 0.8) == (0.4, 0.5)
    assert P.lambda_transform("0.1f", 0.0)[0] == float(np.float32(0.1))
    assert P.lambda_transform("lambda >= 0.5 && lambda < 0.9", 0.6) == (1.0, 0.0)
    assert P.lambda_transform("-(lambda - 2) * 3", 1.0) == (3.0, -3.0)


@pytest.mark.parametrize("bad", ["lambda +", "lamda", "sin(lambda, 2)", "foo(lambda)", "(lambda", "lambda ? 1", ""])
def test_lambda_transform_parse_errors(bad):
    with pytest.raises(RuntimeError, match="lambda transform"):
        P.lambda_transform(bad, 0.5)


def test_plain_nonbonded_refuses_transforms_it_would_drop():
    """The reference's Nonbonded.unbound_impl ignores args[6:]
    (timemachine/lib/potentials.py:284-301); here a non-identity expression
    there raises instead of being dropped (before any device work)."""
    args = (np.array([[0, 1]]), np.ones((1, 2)), [0, 0], [0, 1], 2.0, 1.2)
    with pytest.raises(RuntimeError, match="does not apply lambda transform"):
        P.Nonbonded(*args, "lambda*lambda").unbound_impl(np.float32)
    with pytest.raises(RuntimeError, match="does not apply lambda transform"):
        P.Nonbonded(*args, "lambda", "lambda", "lambda", "1-lambda").unbound_impl(np.float64)
    with pytest.raises(RuntimeError, match="at most 4"):
        P.NonbondedInterpolated(*args, "lambda", "lambda", "lambda", "lambda", "lambda").unbound_impl(np.float32)


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
