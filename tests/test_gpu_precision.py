"""FP64 pair arithmetic, lambda-transform expressions and the reference's
near-coincident exclusion case, on the GPU through the C ABI.

Tolerances are the reference tests' own: FP64 rtol 1e-8 (atol 1e-11 for the
transform test), FP32 rtol 1e-4 (tests/test_parameter_interpolation.py:138,
tests/test_nonbonded.py:402, tests/nonbonded/test_nonbonded_all_pairs.py:133),
with forces compared by max_i |dF_i| / max(|F_i|, 1) (tests/common.py:386-409).
Where the reference CUDA build (oracle/_ref) is present, the FP64 kernels are
also compared with the reference's _f64 kernels.
"""

import itertools

import numpy as np
import pytest
import torch

from oracle.nonbonded_oracle import Oracle, force_error
from oracle.refgpu import refgpu
from tests.gpu_helpers import decode, ref_runner, run_device
from tests.helpers import f32_round, random_params, small_water_case
from tests.test_gpu_parity import CASES, _inputs, _nonbonded
from timemachine_b200 import potentials as P

pytestmark = pytest.mark.gpu

needs_ref = pytest.mark.skipif(not refgpu.available(), reason="reference CUDA build (oracle/_ref) not present")

# force bar (1e-5, relative to max(|F|, 1)) of the FP64 path against the FP64 oracle
FORCE_BAR_F64 = 1e-5


def compare(ref, test, rtol, atol, label="", atol_dp=None):
    """tests/common.py:412-480 compare_forces: u, du_dl, du_dp by allclose, du_dx by the force metric."""
    r_dx, r_dp, r_dl, r_u = ref
    t_dx, t_dp, t_dl, t_u = test
    ef = force_error(r_dx, t_dx)
    assert ef <= rtol, f"{label} du_dx {ef:.3e}"
    np.testing.assert_allclose(t_u, r_u, rtol=rtol, atol=atol, err_msg=f"{label} u")
    np.testing.assert_allclose(t_dl, r_dl, rtol=rtol, atol=max(atol, 1e-12), err_msg=f"{label} du_dl")
    atol_dp = atol if atol_dp is None else atol_dp
    np.testing.assert_allclose(t_dp, r_dp.reshape(t_dp.shape), rtol=rtol, atol=atol_dp, err_msg=f"{label} du_dp")
    return ef


@pytest.mark.parametrize("name", ["water3k", "random231", "random1050", "golden_repro", "golden_bad_test_547"])
def test_f64_vs_fp64_oracle(name):
    """The FP64 kernels against the FP64 oracle: every output within the
    reference's FP64 tolerance, forces far inside the 1e-5 bar."""
    c = CASES[name]()
    x, p, box = _inputs(c)
    mine = _nonbonded(c).unbound_impl(np.float64)
    test = decode(run_device(mine, x, p, box, c["lam"]), p.shape)
    o = Oracle(c["plane"], c["offset"], c["beta"], c["cutoff"], c["exclusion_idxs"], c["scales"], c["interpolated"])
    ref = o(x, p, box, c["lam"])
    ef = compare(ref, test, 1e-8, 1e-8, name)
    print(f"\n[{name}] FP64 force error {ef:.2e}")
    assert ef < FORCE_BAR_F64


def test_f64_every_output_selection_and_determinism():
    """All 16 output selections of the FP64 kernels equal the full evaluation's
    outputs bit for bit, and a second run repeats them."""
    c = CASES["random231"]()
    x, p, box = _inputs(c)
    mine = _nonbonded(c).unbound_impl(np.float64)
    full = run_device(mine, x, p, box, c["lam"])
    for combo in itertools.product([False, True], repeat=4):
        a = run_device(mine, x, p, box, c["lam"], *combo)
        b = run_device(mine, x, p, box, c["lam"], *combo)
        for k in range(4):
            if combo[k]:
                np.testing.assert_array_equal(a[k], full[k])
                np.testing.assert_array_equal(a[k], b[k])
            else:
                assert a[k] is None


@needs_ref
@pytest.mark.parametrize("name", ["water3k", "random231", "golden_repro"])
def test_f64_vs_reference_f64_kernel(name):
    """The FP64 kernels against the reference's _f64 kernels on the same
    inputs. Both round each pair's FP64 terms into the same int64 fixed point;
    the force, du_dp, du_dl and energy sums agree to the FP64 tolerance, and
    the fraction of bit-identical entries is reported."""
    c = CASES[name]()
    x, p, box = _inputs(c)
    mine = _nonbonded(c).unbound_impl(np.float64)
    ref = refgpu.RefNonbonded(c["exclusion_idxs"], c["scales"], c["plane"], c["offset"], c["beta"], c["cutoff"],
                              c["interpolated"], precision=64)
    a = run_device(mine, x, p, box, c["lam"])
    b = run_device(ref, x, p, box, c["lam"], runner=ref_runner)
    same = [float(np.mean(np.asarray(a[k]).ravel() == np.asarray(b[k]).ravel())) for k in range(4)]
    print(f"\n[{name}] bit-identical fraction vs reference _f64: du_dx {same[0]:.4f} du_dp {same[1]:.4f} "
          f"du_dl {same[2]:.0f} u {same[3]:.0f}")
    compare(decode(b, p.shape), decode(a, p.shape), 1e-8, 1e-9, name)


def test_f64_multi_window_equals_single_windows():
    """K FP64 windows in one call equal K single-window calls bit for bit."""
    c = CASES["random1050"]()
    x, p, box = _inputs(c)
    impl = _nonbonded(c).unbound_impl(np.float64)
    lams = np.linspace(0.0, 1.0, 5)
    mdx, mdp, mdl, mu = impl.execute_windows_fixed(x, p, box, lams)
    single = _nonbonded(c).unbound_impl(np.float64)
    for k, lam in enumerate(lams):
        sdx, sdp, sdl, su = single._execute_fixed(x, p, box, lam, True, True, True, True)
        np.testing.assert_array_equal(mdx[k], sdx)
        np.testing.assert_array_equal(mdp[k], sdp)
        assert mdl[k].sum(dtype=np.uint64) == sdl.sum(dtype=np.uint64)
        assert mu[k].sum(dtype=np.uint64) == su.sum(dtype=np.uint64)


# tests/test_parameter_interpolation.py:91-140: the four transforms and their jax forms
TRANSFORM_EXPRS = ["lambda*lambda", "sin(lambda*PI/2)", "lambda < 0.5 ? sin(lambda*PI)*sin(lambda*PI) : 1",
                   "1-lambda*lambda"]
TRANSFORM_FNS = (
    lambda l: l * l,
    lambda l: torch.sin(l * np.pi / 2),
    lambda l: torch.where(l < 0.5, torch.sin(l * np.pi) * torch.sin(l * np.pi), torch.ones_like(l)),
    lambda l: 1 - l * l,
)


def _advanced_case():
    """36 water atoms in a 3 nm box, cutoff 1.0, random planes/offsets in
    {0, 1}, two parameter sets (sigma scale 5), as the reference test builds it."""
    rng = np.random.default_rng(4321)
    c = small_water_case(rng, 36, planes=(0, 2), offsets=(0, 2))
    src = c["params"]
    dst = random_params(rng, src.shape[0], 5.0)
    return c, np.concatenate([src, dst])


# FP32 du_dp: an entry that is a small remainder of large cancelling pair terms
# (0.011 out of terms of order 100) carries an FP32 rounding error of a few
# 1e-6, so its absolute tolerance is 1e-5 (measured: 4.5e-6 on one of 216).
@pytest.mark.parametrize("precision,rtol,atol,atol_dp", [(np.float64, 1e-8, 1e-11, 1e-11),
                                                         (np.float32, 1e-4, 1e-6, 1e-5)])
def test_lambda_transforms_vs_oracle(precision, rtol, atol, atol_dp):
    """NonbondedInterpolated with the reference test's four transform
    expressions, at its six lambdas and for every output selection, against
    the FP64 oracle evaluating the same transforms (autograd through them)."""
    c, qlj = _advanced_case()
    x, p = f32_round(c["x"]), f32_round(qlj)
    box = np.eye(3) * 3.0
    pot = P.NonbondedInterpolated(c["exclusion_idxs"], c["scales"], c["plane"], c["offset"], 2.0, 1.0,
                                  *TRANSFORM_EXPRS)
    impl = pot.unbound_impl(precision)
    o = Oracle(c["plane"], c["offset"], 2.0, 1.0, c["exclusion_idxs"], c["scales"], interpolated=True,
               transforms=TRANSFORM_FNS)
    for lam in [0.0, 0.2, 0.6, 0.7, 0.8, 1.0]:
        ref = o(x, p, box, lam)
        test = impl.execute(x, p, box, lam)
        compare(ref, test, rtol, atol, f"lambda={lam}", atol_dp)
        for combo in itertools.product([False, True], repeat=4):
            sel = impl.execute_selective(x, p, box, lam, *combo)
            for k in range(4):
                if combo[k]:
                    np.testing.assert_array_equal(sel[k], test[k])


def test_lambda_transforms_change_the_result_and_windows_agree():
    """Transforms are applied (a non-identity w schedule moves du_dl and u
    away from the identity's), and a multi-window call with transforms equals
    single-window calls bit for bit."""
    c, qlj = _advanced_case()
    x, p = f32_round(c["x"]), f32_round(qlj)
    box = np.eye(3) * 3.0
    args = (c["exclusion_idxs"], c["scales"], c["plane"], c["offset"], 2.0, 1.0)
    with_t = P.NonbondedInterpolated(*args, *TRANSFORM_EXPRS).unbound_impl(np.float32)
    ident = P.NonbondedInterpolated(*args).unbound_impl(np.float32)
    a = with_t.execute(x, p, box, 0.3)
    b = ident.execute(x, p, box, 0.3)
    assert a[3] != b[3] and a[2] != b[2]
    lams = np.array([0.0, 0.3, 0.55, 0.9])
    mdx, mdp, mdl, mu = with_t.execute_windows_fixed(x, p, box, lams)
    single = P.NonbondedInterpolated(*args, *TRANSFORM_EXPRS).unbound_impl(np.float32)
    for k, lam in enumerate(lams):
        sdx, sdp, sdl, su = single._execute_fixed(x, p, box, lam, True, True, True, True)
        np.testing.assert_array_equal(mdx[k], sdx)
        np.testing.assert_array_equal(mdp[k], sdp)
        assert mdl[k].sum(dtype=np.uint64) == sdl.sum(dtype=np.uint64)
        assert mu[k].sum(dtype=np.uint64) == su.sum(dtype=np.uint64)


@needs_ref
def test_lambda_transforms_vs_reference_kernel():
    """The same transforms through the reference build (its run-time compiled
    transforms): FP32 outputs within the FP32 tolerance of the reference's, and
    du_dx bit-identical (the transforms only move w and the parameters, whose
    FP32 staging rounds the same)."""
    c, qlj = _advanced_case()
    x, p = f32_round(c["x"]), f32_round(qlj)
    box = np.eye(3) * 3.0
    mine = P.NonbondedInterpolated(c["exclusion_idxs"], c["scales"], c["plane"], c["offset"], 2.0, 1.0,
                                   *TRANSFORM_EXPRS).unbound_impl(np.float32)
    ref = refgpu.RefNonbonded(c["exclusion_idxs"], c["scales"], c["plane"], c["offset"], 2.0, 1.0, True,
                              transforms=TRANSFORM_EXPRS)
    for lam in [0.0, 0.2, 0.6, 1.0]:
        a = run_device(mine, x, p, box, lam)
        b = run_device(ref, x, p, box, lam, runner=ref_runner)
        np.testing.assert_array_equal(a[0], b[0])
        compare(decode(b, p.shape), decode(a, p.shape), 1e-6, 1e-8, f"lambda={lam}")


def _coincident_case():
    """tests/test_nonbonded.py:344-406: 126 water atoms in a 3 nm box; ten
    atoms, mutually excluded at full scale, all moved to within 1e-3 nm of
    (2, 2, 2), so their pair terms are huge and must cancel exactly against
    the exclusions in fixed point."""
    rng = np.random.default_rng(2020)
    c = small_water_case(rng, 126)
    x = c["x"].copy()
    N = x.shape[0]
    ex_atoms = rng.choice(np.arange(N), size=10, replace=False)
    excl = np.array([(i, j) for a, i in enumerate(ex_atoms) for b, j in enumerate(ex_atoms) if b > a], np.int32)
    scales = np.ones((len(excl), 2))
    for i in ex_atoms:
        x[i] = np.zeros(3) + rng.random() / 1000 + 2
    plane = rng.integers(0, 2, size=N, dtype=np.int32)
    offset = rng.integers(0, 2, size=N, dtype=np.int32)
    return x, c["params"], np.eye(3) * 3.0, excl, scales, plane, offset


# FP32 du_dl of this case: the reference's FP32 arithmetic (reproduced bit for
# bit, see the next test) overflows to -inf in the LJ prefactor of coincident
# pairs, and in a tile that holds a lambda-dependent atom the du_dl term of a
# pair with delta_w = 0 becomes 0 * inf = NaN, which the fixed-point
# conversion saturates to -2^63; the exclusion pass skips du_dl for pairs of
# two lambda-independent atoms (timemachine/cpp/src/kernels/k_nonbonded_pair_list.cuh:208),
# so one such term is left: du_dl = -2^63 / 2^36 = -2^27. The FP64 path has no
# overflow and matches the oracle's 0.
SATURATED_DU_DL = -(2.0**27)


@pytest.mark.parametrize("precision,rtol", [(np.float64, 1e-8), (np.float32, 1e-4)])
def test_near_coincident_exclusions_cancel(precision, rtol):
    x, params, box, excl, scales, plane, offset = _coincident_case()
    x, params = f32_round(x), f32_round(params)
    impl = P.Nonbonded(excl, scales, plane, offset, 2.0, 1.0).unbound_impl(precision)
    o = Oracle(plane, offset, 2.0, 1.0, excl, scales)
    ref = o(x, params, box, 0.0)
    full = impl.execute(x, params, box, 0.0)
    for combo in itertools.product([False, True], repeat=4):
        out = impl.execute_selective(x, params, box, 0.0, *combo)
        for k in range(4):
            if combo[k]:
                np.testing.assert_array_equal(out[k], full[k])
    if precision == np.float32:
        assert full[2] in (SATURATED_DU_DL, pytest.approx(ref[2], rel=rtol, abs=1e-8)), full[2]
        full = (full[0], full[1], ref[2], full[3])
    compare(ref, full, rtol, 1e-8, "coincident")


@needs_ref
@pytest.mark.parametrize("precision", [32, 64])
def test_near_coincident_exclusions_bitexact_vs_reference(precision):
    """The saturated fixed-point conversions of the coincident pairs, and
    their cancellation, match the reference kernels bit for bit (FP32) or in
    the outputs' sums (FP64)."""
    x, params, box, excl, scales, plane, offset = _coincident_case()
    x, params = f32_round(x), f32_round(params)
    mine = P.Nonbonded(excl, scales, plane, offset, 2.0, 1.0).unbound_impl(
        np.float64 if precision == 64 else np.float32)
    ref = refgpu.RefNonbonded(excl, scales, plane, offset, 2.0, 1.0, False, precision=precision)
    a = run_device(mine, x, params, box, 0.0)
    b = run_device(ref, x, params, box, 0.0, runner=ref_runner)
    if precision == 32:
        for k in range(4):
            np.testing.assert_array_equal(a[k], b[k])
    else:
        compare(decode(b, params.shape), decode(a, params.shape), 1e-8, 1e-9, "coincident f64")


def _np_decode(fixed, p_shape):
    from timemachine_b200.fixed_point import du_dp_fixed_to_float, fixed_to_float, sum_fixed

    dx, dp, dl, u = fixed
    return fixed_to_float(dx), du_dp_fixed_to_float(dp).reshape(p_shape), fixed_to_float(sum_fixed(dl)), \
        fixed_to_float(sum_fixed(u))


@pytest.mark.parametrize("interpolated", [False, True])
def test_f64_pair_list_and_group_vs_oracle(interpolated):
    """The FP64 kernels of the other potentials of the path: the negated pair
    list (exclusions) and the interaction group, plain and interpolated,
    within the reference's FP64 tolerance of the oracle."""
    from oracle.nonbonded_oracle import interaction_group_oracle, pair_list_oracle

    rng = np.random.default_rng(77 + int(interpolated))
    c = small_water_case(rng, 400)
    N = c["x"].shape[0]
    params = c["params"]
    if interpolated:
        params = np.concatenate([params, params * rng.uniform(0.5, 1.5, size=params.shape)])
    x, p, box = f32_round(c["x"]), f32_round(params), c["box"]
    lam = 0.35
    cls = P.NonbondedPairListNegatedInterpolated if interpolated else P.NonbondedPairListNegated
    pl = cls(c["exclusion_idxs"], c["scales"], c["plane"], c["offset"], 2.0, 1.0).unbound_impl(np.float64)
    test = pl.execute(x, p, box, lam)
    rx, rp, rl, ru = pair_list_oracle(x, p, box, lam, c["plane"], c["offset"], 2.0, 1.0, c["exclusion_idxs"],
                                      c["scales"], interpolated)
    compare((-rx, -rp, -rl, -ru), test, 1e-8, 1e-8, "pair list")
    rows = rng.choice(N, size=37, replace=False).astype(np.int32)
    gcls = P.NonbondedInteractionGroupInterpolated if interpolated else P.NonbondedInteractionGroup
    g = gcls(rows, c["plane"], c["offset"], 2.0, 1.1).unbound_impl(np.float64)
    test = g.execute(x, p, box, lam)
    ref = interaction_group_oracle(x, p, box, lam, c["plane"], c["offset"], 2.0, 1.1, rows, interpolated)
    compare(ref, test, 1e-8, 1e-8, "group")


@needs_ref
@pytest.mark.parametrize("interpolated", [False, True])
def test_f64_group_vs_reference_f64_kernel(interpolated):
    from timemachine_b200 import testsystems

    rng = np.random.default_rng(91)
    s = testsystems.build_system(700, 3.0, seed=21, n_ligand=24)
    rows = np.flatnonzero(s.lambda_offset_idxs != 0).astype(np.int32)
    params = s.params
    if interpolated:
        params = np.concatenate([params, params * rng.uniform(0.8, 1.2, size=params.shape)])
    x, p = f32_round(s.x), f32_round(params)
    gcls = P.NonbondedInteractionGroupInterpolated if interpolated else P.NonbondedInteractionGroup
    mine = gcls(rows, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff).unbound_impl(np.float64)
    ref = refgpu.RefInteractionGroup(rows, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff,
                                     interpolated, precision=64)
    for lam in [0.0, 0.4]:
        a = mine._execute_fixed(x, p, s.box, lam, True, True, True, True)
        b = ref.execute_host_fixed(x, p, s.box, lam)
        compare(_np_decode(b, p.shape), _np_decode(a, p.shape), 1e-8, 1e-9, f"group lambda={lam}")


def test_lambda_transforms_on_the_interaction_group():
    """The group forwards the transform expressions too (its constructor's
    last four arguments), checked against the oracle with the same transforms."""
    from oracle.nonbonded_oracle import interaction_group_oracle

    c, qlj = _advanced_case()
    x, p = f32_round(c["x"]), f32_round(qlj)
    box = np.eye(3) * 3.0
    rows = np.arange(0, 36, 3, dtype=np.int32)
    g = P.NonbondedInteractionGroupInterpolated(rows, c["plane"], c["offset"], 2.0, 1.0,
                                                *TRANSFORM_EXPRS).unbound_impl(np.float64)
    for lam in [0.1, 0.6]:
        test = g.execute(x, p, box, lam)
        ref = interaction_group_oracle(x, p, box, lam, c["plane"], c["offset"], 2.0, 1.0, rows, True,
                                       transforms=TRANSFORM_FNS)
        compare(ref, test, 1e-8, 1e-11, f"lambda={lam}", 1e-11)
