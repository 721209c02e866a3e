"""GPU tests of the multi-window evaluation (K lambda windows in one launch
sequence): every window's raw int64 outputs equal a single-window evaluation
at that lambda, bit for bit, for each potential kind and output selection.

The reference evaluates windows one at a time (execute_selective_batch,
timemachine/cpp/src/wrap_kernels.cpp:381-551; Context::multiple_steps_U,
timemachine/cpp/src/context.cu:139-209); fixed-point accumulation makes the
shared-tile evaluation order-independent, so equality is exact.
"""

import itertools

import numpy as np
import pytest
import torch

from oracle.refgpu import refgpu
from tests.conftest import load_golden
from tests.gpu_helpers import to_dev
from tests.helpers import small_water_case
from timemachine_b200 import _lib
from timemachine_b200 import potentials as P
from timemachine_b200 import testsystems

pytestmark = pytest.mark.gpu

LAMBDAS_12 = np.array([0.0, 0.02, 0.05, 0.1, 0.2, 0.3, 0.45, 0.5, 0.6, 0.75, 0.9, 1.0])


def _single(impl, x, p, box, lams, flags=(True, True, True, True)):
    outs = [impl._execute_fixed(x, p, box, lam, *flags) for lam in lams]
    return [None if outs[0][c] is None else np.stack([o[c] for o in outs]) for c in range(4)]


def _assert_windows_equal(impl, x, p, box, lams, flags=(True, True, True, True)):
    multi = impl.execute_windows_fixed(x, p, box, lams, *flags)
    single = _single(impl, x, p, box, lams, flags)
    for c, name in enumerate(["du_dx", "du_dp", "du_dl", "u"]):
        if not flags[c]:
            assert multi[c] is None
            continue
        np.testing.assert_array_equal(multi[c], single[c], err_msg=name)
    return multi


def _ligand_system():
    s = testsystems.build_system(700, 3.0, seed=21, n_ligand=24)
    assert np.any(s.lambda_offset_idxs != 0)
    return s


def test_nonbonded_windows_equal_single_window():
    s = _ligand_system()
    impl = P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    impl = impl.unbound_impl(np.float32)
    multi = _assert_windows_equal(impl, s.x, s.params, s.box, LAMBDAS_12)
    # the windows do differ (the ligand decouples along w)
    u = multi[3].view(np.int64).sum(axis=1)
    assert len(set(u.tolist())) > 1


@pytest.mark.parametrize("name", ["repro", "bad_test_547"])
def test_interpolated_windows_equal_single_window(name):
    g = load_golden(name)
    impl = P.NonbondedInterpolated(
        g["exclusion_idxs"], g["scales"], g["lambda_plane_idxs"], g["lambda_offset_idxs"], g["beta"], g["cutoff"]
    ).unbound_impl(np.float32)
    lams = np.array([0.0, float(g["lam"]), 0.33, 0.5, 1.0])
    _assert_windows_equal(impl, g["x"], g["params"], g["box"], lams)
    # forces only and energy only: the packed two-rows sweep, per-window units included
    _assert_windows_equal(impl, g["x"], g["params"], g["box"], lams, (True, False, False, False))
    _assert_windows_equal(impl, g["x"], g["params"], g["box"], lams, (False, False, False, True))


def test_windows_follow_changed_lambda_dependence_without_rebuild():
    """Interpolated parameters decide which atoms are lambda-dependent (p0 !=
    p1). A multi-window call keeps its list of lambda-dependent tiles across
    calls; when new parameters change that set while the atoms stay put (no
    neighbour-list rebuild), the list must be redone: the windows equal a
    fresh potential's."""
    s = _ligand_system()
    make = lambda: P.NonbondedInterpolated(
        s.exclusion_idxs, s.scales, s.lambda_plane_idxs, np.zeros_like(s.lambda_offset_idxs), s.beta, s.cutoff
    ).unbound_impl(np.float32)
    lig = np.flatnonzero(s.lambda_offset_idxs != 0)
    p_a = np.concatenate([s.params, s.params])
    p_a[s.N + lig[: lig.size // 2], 0] *= 0.5  # first half of the ligand's charges change with lambda
    p_b = np.concatenate([s.params, s.params])
    p_b[s.N + lig[lig.size // 2 :], 0] *= 0.5  # now the other half
    lams = np.linspace(0.0, 1.0, 6)
    impl = make()
    impl.execute_windows_fixed(s.x, p_a, s.box, lams)
    rebuilds = impl.nblist_stats()[2]
    got = impl.execute_windows_fixed(s.x, p_b, s.box, lams)
    assert impl.nblist_stats()[2] == rebuilds  # same list, new lambda dependence
    want = make().execute_windows_fixed(s.x, p_b, s.box, lams)
    for c in (0, 1):
        np.testing.assert_array_equal(got[c], want[c])
    for c in (2, 3):
        np.testing.assert_array_equal(got[c].sum(axis=1, dtype=np.uint64), want[c].sum(axis=1, dtype=np.uint64))
    single = _single(impl, s.x, p_b, s.box, lams)
    np.testing.assert_array_equal(got[0], single[0])


def test_all_pairs_subset_and_pair_list_windows():
    rng = np.random.default_rng(2022)
    c = small_water_case(rng, 600)
    N = c["x"].shape[0]
    atom_idxs = rng.choice(N, size=N // 3, replace=False).astype(np.int32)
    lams = np.linspace(0.0, 1.0, 7)
    ap = P.NonbondedAllPairsInterpolated(c["plane"], c["offset"], 2.0, 1.0, atom_idxs).unbound_impl(np.float32)
    p2 = np.concatenate([c["params"], c["params"] * 1.1])
    _assert_windows_equal(ap, c["x"], p2, c["box"], lams)
    pl = P.NonbondedPairListNegated(c["exclusion_idxs"], c["scales"], c["plane"], c["offset"], 2.0, 1.0)
    _assert_windows_equal(pl.unbound_impl(np.float32), c["x"], c["params"], c["box"], lams)


def test_every_output_selection():
    s = _ligand_system()
    impl = P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    impl = impl.unbound_impl(np.float32)
    lams = np.array([0.1, 0.6, 0.95])
    for flags in itertools.product([False, True], repeat=4):
        if not any(flags):
            continue
        _assert_windows_equal(impl, s.x, s.params, s.box, lams, flags)


def test_window_count_limits():
    s = testsystems.build_system(400, 2.8, seed=3, n_ligand=8)
    impl = P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    impl = impl.unbound_impl(np.float32)
    _assert_windows_equal(impl, s.x, s.params, s.box, np.linspace(0, 1, 32))
    _assert_windows_equal(impl, s.x, s.params, s.box, np.array([0.4]))
    with pytest.raises(_lib.TmnbError, match="number of lambda windows must be in"):
        impl.execute_windows_fixed(s.x, s.params, s.box, np.linspace(0, 1, 33))


def test_selective_batch_crosses_window_chunks():
    """40 lambdas (two multi-window evaluations) x 2 coordinate sets x 2 parameter sets."""
    s = testsystems.build_system(400, 2.8, seed=4, n_ligand=8)
    impl = P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    impl = impl.unbound_impl(np.float32)
    rng = np.random.default_rng(5)
    xs = np.stack([s.x, s.x + rng.normal(scale=0.01, size=s.x.shape)])
    ps = np.stack([s.params, s.params * 0.9])
    boxes = np.stack([s.box, s.box])
    lams = np.linspace(0.0, 1.0, 40)
    du_dx, du_dp, du_dl, u = impl.execute_selective_batch(xs, ps, boxes, lams, True, True, True, True)
    assert du_dx.shape == (2, 2, 40, s.N, 3) and u.shape == (2, 2, 40)
    for ci, pi, li in [(0, 0, 0), (1, 0, 31), (0, 1, 32), (1, 1, 39)]:
        ref = impl.execute_selective(xs[ci], ps[pi], boxes[ci], lams[li], True, True, True, True)
        np.testing.assert_array_equal(du_dx[ci, pi, li], ref[0])
        np.testing.assert_array_equal(du_dp[ci, pi, li], ref[1])
        assert du_dl[ci, pi, li] == ref[2]
        assert u[ci, pi, li] == ref[3]


def test_device_windows_accumulate_and_interleave_with_single_calls():
    s = _ligand_system()
    impl = P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    impl = impl.unbound_impl(np.float32)
    K, N = 6, s.N
    lams = np.linspace(0.0, 1.0, K)
    x, p, box = to_dev(s.x), to_dev(s.params).reshape(-1), to_dev(s.box)
    du_dx = torch.zeros((K, N, 3), dtype=torch.int64, device="cuda")
    u = torch.zeros((K, N), dtype=torch.int64, device="cuda")
    impl.execute_windows_device(x, p, box, lams, du_dx=du_dx, u=u)
    # a single-window call in between (same neighbour list) must not disturb the next multi-window call
    one = torch.zeros((N, 3), dtype=torch.int64, device="cuda")
    impl.execute_device(x, p, box, 0.3, du_dx=one)
    impl.execute_windows_device(x, p, box, lams, du_dx=du_dx, u=u)
    impl.check_device_error()
    torch.cuda.synchronize()
    single = _single(impl, s.x, s.params, s.box, lams, (True, False, False, True))
    np.testing.assert_array_equal(du_dx.cpu().numpy().view(np.uint64), single[0] * np.uint64(2))
    np.testing.assert_array_equal(u.cpu().numpy().view(np.uint64), single[3] * np.uint64(2))


@pytest.mark.skipif(not refgpu.available(), reason="reference build (oracle/_ref) not present")
def test_windows_bitexact_against_reference_build():
    """Each window of one multi-window evaluation equals the reference CUDA
    kernel at that lambda (23k-atom box with a decoupling ligand)."""
    s = testsystems.water_ligand_23k()
    impl = P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    impl = impl.unbound_impl(np.float32)
    ref = refgpu.RefNonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    lams = np.array([0.0, 0.25, 0.5, 1.0])
    mdx, mdp, mdl, mu = impl.execute_windows_fixed(s.x, s.params, s.box, lams)
    for k, lam in enumerate(lams):
        rdx, rdp, rdl, ru = ref.execute_host_fixed(s.x, s.params, s.box, lam)
        np.testing.assert_array_equal(mdx[k], rdx)
        np.testing.assert_array_equal(mdp[k], rdp)
        assert mdl[k].sum(dtype=np.uint64) == rdl.sum(dtype=np.uint64)
        assert mu[k].sum(dtype=np.uint64) == ru.sum(dtype=np.uint64)
