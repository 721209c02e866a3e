"""Fixed-point decoding of the int64 accumulators.

timemachine/cpp/src/fixed_point.hpp:3-17: value = (double)(int64)bits / 2^e with
e = 36 for du_dx, u, du_dl and du_dcharge, 37 for du_dsigma, 38 for
du_depsilon. Per-atom u/du_dl buffers are summed as uint64 (wrapping, exactly
as std::accumulate over unsigned long long) before decoding.
"""

import numpy as np

FIXED_EXPONENT = 2**36
FIXED_EXPONENT_DU_DCHARGE = 2**36
FIXED_EXPONENT_DU_DSIG = 2**37
FIXED_EXPONENT_DU_DEPS = 2**38


def fixed_to_float(v, exponent=FIXED_EXPONENT):
    """Decode uint64 (or int64) fixed-point values to float64."""
    a = np.asarray(v)
    if a.dtype == np.uint64:
        a = a.view(np.int64)
    if a.ndim == 0:
        return float(np.int64(a)) / exponent
    return a.astype(np.float64) / exponent


def sum_fixed(v):
    """Wrapping uint64 sum of a per-atom fixed-point buffer."""
    a = np.asarray(v, dtype=np.uint64)
    with np.errstate(over="ignore"):
        return np.uint64(a.sum(dtype=np.uint64))


def du_dp_fixed_to_float(du_dp):
    """Per-column exponents of [..., 3] parameter derivatives
    (timemachine/cpp/src/nonbonded_all_pairs.cu:435-450)."""
    a = np.asarray(du_dp, dtype=np.uint64).reshape(-1, 3).view(np.int64).astype(np.float64)
    a[:, 0] /= FIXED_EXPONENT_DU_DCHARGE
    a[:, 1] /= FIXED_EXPONENT_DU_DSIG
    a[:, 2] /= FIXED_EXPONENT_DU_DEPS
    return a.reshape(np.asarray(du_dp).shape)
