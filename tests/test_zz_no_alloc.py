"""GPU test of tmnb_pair_list_execute_static, the allocation-free pair-list
entry point (no reference counterpart): two calls in a row on caller-owned
device buffers give the outputs of the allocating entry point
(tmnb_pair_list_create + tmnb_potential_execute_device) within tolerance,
and sizes beyond TMNB_STATIC_MAX_ATOMS are rejected.

This file is named so that pytest collects it last; it passes alone and after
the other GPU tests.
"""

import ctypes

import numpy as np
import pytest
import torch

from tests.helpers import small_water_case
from timemachine_b200 import _lib
from timemachine_b200 import potentials as P

pytestmark = pytest.mark.gpu

STATIC_MAX_ATOMS = 32768
# Both paths run the same per-pair FP32 arithmetic and int64 fixed-point sums,
# so they agree exactly; the tolerance on the decoded values is stated anyway.
RTOL = 1e-9
ATOL_FIXED = 0


def _dev(a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _addr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _case(negated):
    rng = np.random.default_rng(20241 + int(negated))
    c = small_water_case(rng, 1500)
    return c


def _allocating(c, negated, lam, outs):
    cls = P.NonbondedPairListNegated if negated else P.NonbondedPairList
    impl = cls(c["exclusion_idxs"], c["scales"], c["plane"], c["offset"], 2.0, 1.0).unbound_impl(np.float32)
    x, p, box = _dev(c["x"], torch.float64), _dev(c["params"], torch.float64).reshape(-1), _dev(c["box"], torch.float64)
    impl.execute_device(x, p, box, lam, *outs)
    torch.cuda.synchronize()


def _static(c, negated, lam, outs):
    lib = _lib.lib()
    N = c["x"].shape[0]
    pairs = _dev(np.asarray(c["exclusion_idxs"]).reshape(-1, 2), torch.int32)
    scales = _dev(np.asarray(c["scales"]).reshape(-1, 2), torch.float64)
    plane = _dev(c["plane"], torch.int32)
    offset = _dev(c["offset"], torch.int32)
    x, p, box = _dev(c["x"], torch.float64), _dev(c["params"], torch.float64), _dev(c["box"], torch.float64)
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(
        lib.tmnb_pair_list_execute_static(
            N, pairs.shape[0], _addr(pairs), _addr(scales), _addr(plane), _addr(offset), 2.0, 1.0,
            1 if negated else 0, _addr(x), _addr(p), _addr(box), float(lam), *[_addr(o) for o in outs],
            ctypes.c_void_p(stream),
        )
    )
    torch.cuda.synchronize()


def _zeros(N):
    return [torch.zeros(sh, dtype=torch.int64, device="cuda") for sh in [(N, 3), (N * 3,), (N,), (N,)]]


def _decoded(outs):
    from timemachine_b200.fixed_point import du_dp_fixed_to_float, fixed_to_float, sum_fixed

    dx, dp, dl, u = [o.cpu().numpy().view(np.uint64) for o in outs]
    return fixed_to_float(dx), du_dp_fixed_to_float(dp), fixed_to_float(sum_fixed(dl)), fixed_to_float(sum_fixed(u))


@pytest.mark.parametrize("negated", [False, True])
def test_static_entry_matches_allocating_entry_on_two_calls_in_a_row(negated):
    c = _case(negated)
    N = c["x"].shape[0]
    for call, lam in enumerate([0.3, 0.7]):
        ref = _zeros(N)
        _allocating(c, negated, lam, ref)
        got = _zeros(N)
        _static(c, negated, lam, got)
        for name, r, g in zip(["du_dx", "du_dp", "du_dl", "u"], ref, got):
            r_raw, g_raw = r.cpu().numpy(), g.cpu().numpy()
            assert np.max(np.abs(r_raw - g_raw)) <= ATOL_FIXED, (call, name)
        for name, r, g in zip(["du_dx", "du_dp", "du_dl", "u"], _decoded(ref), _decoded(got)):
            np.testing.assert_allclose(g, r, rtol=RTOL, atol=0, err_msg=f"call {call} {name}")
        assert np.any(got[0].cpu().numpy() != 0)


def test_static_entry_subset_of_outputs():
    c = _case(False)
    N = c["x"].shape[0]
    ref = _zeros(N)
    _allocating(c, False, 0.5, ref)
    got = [torch.zeros((N, 3), dtype=torch.int64, device="cuda"), None, None, torch.zeros(N, dtype=torch.int64, device="cuda")]
    _static(c, False, 0.5, got)
    np.testing.assert_array_equal(got[0].cpu().numpy(), ref[0].cpu().numpy())
    np.testing.assert_array_equal(got[3].cpu().numpy(), ref[3].cpu().numpy())


def test_static_entry_rejects_sizes_beyond_capacity():
    lib = _lib.lib()
    N = STATIC_MAX_ATOMS + 1
    rc = lib.tmnb_pair_list_execute_static(
        N, 0, None, None, None, None, 2.0, 1.0, 0, None, None, None, 0.0, None, None, None, None, None
    )
    assert rc == 1  # TMNB_ERR_INVALID_ARGUMENT
    msg = lib.tmnb_last_error().decode()
    assert "exceeds the static scratch capacity of 32768 atoms" in msg


def test_static_entry_reports_bad_pairs_and_recovers():
    """A pair index outside [0, N) or a pair with src == dst is found on the
    device and returned as TMNB_ERR_INVALID_ARGUMENT with the outputs left
    unchanged (the pair kernel returns before reading any pair); the next
    valid call starts clean and matches the allocating entry point."""
    lib = _lib.lib()
    c = _case(False)
    N = c["x"].shape[0]
    stream = torch.cuda.current_stream().cuda_stream
    for bad in ([[0, N], [1, 2]], [[3, 3], [1, 2]]):
        pairs = _dev(np.asarray(bad), torch.int32)
        scales = _dev(np.ones((2, 2)), torch.float64)
        plane = _dev(c["plane"], torch.int32)
        offset = _dev(c["offset"], torch.int32)
        x, p, box = _dev(c["x"], torch.float64), _dev(c["params"], torch.float64), _dev(c["box"], torch.float64)
        outs = _zeros(N)
        rc = lib.tmnb_pair_list_execute_static(
            N, 2, _addr(pairs), _addr(scales), _addr(plane), _addr(offset), 2.0, 1.0, 0, _addr(x), _addr(p),
            _addr(box), 0.4, *[_addr(o) for o in outs], ctypes.c_void_p(stream),
        )
        torch.cuda.synchronize()
        assert rc == 1  # TMNB_ERR_INVALID_ARGUMENT
        assert "pair index out of range [0, N) or src == dst" in lib.tmnb_last_error().decode()
        for o in outs:
            assert not torch.any(o != 0)
    ref = _zeros(N)
    _allocating(c, False, 0.4, ref)
    got = _zeros(N)
    _static(c, False, 0.4, got)
    for r, g in zip(ref, got):
        np.testing.assert_array_equal(g.cpu().numpy(), r.cpu().numpy())
