"""GPU parity of the B200 nonbonded potential (through the C ABI).

Two tiers, as the reference's fixed-point design allows:
  1. bit-exact int64 accumulators against the reference CUDA kernel built from
     the reference sources (oracle/_ref), when that build is present;
  2. tolerance against the FP64 oracle (restated jax nonbonded_v3), with the
     tolerance written in each test.
Plus the reference's bitwise invariants (determinism, Hilbert on/off, rebuild
cadence, fused vs separate potentials) and its error messages.
"""

import itertools

import numpy as np
import pytest
import torch

from oracle.nonbonded_oracle import Oracle, force_error, pair_list_oracle, rel_error
from oracle.refgpu import refgpu
from tests.conftest import load_golden
from tests.gpu_helpers import decode, ref_runner, run_device
from tests.helpers import f32_round, small_water_case
from timemachine_b200 import potentials as P
from timemachine_b200 import testsystems

pytestmark = pytest.mark.gpu

# Tolerances against the FP64 oracle (inputs rounded through float32 first, as
# tests/common.py:437-438 does). The force metric is max_i |dF_i| / max(|F_i|, 1)
# (tests/common.py:386-409). The reference kernel's own FP32 arithmetic (A&S
# erfc, FP32 per-pair rounding) reaches 5.7e-5 on the water boxes, so the
# bar is the reference tests' float32 tolerance (tests/test_nonbonded.py:199),
# and where the reference build is present the error must equal its error.
TOL_FORCE_WATER = 1e-4
TOL_ENERGY_WATER = 1e-5
TOL_RANDOM = 1e-4


def _case_water3k():
    s = testsystems.water_box_3k()
    return dict(
        x=s.x, params=s.params, box=s.box, exclusion_idxs=s.exclusion_idxs, scales=s.scales,
        plane=s.lambda_plane_idxs, offset=s.lambda_offset_idxs, lam=0.0, beta=s.beta, cutoff=s.cutoff,
        interpolated=False, water=True,
    )


def _case_water23k(lam=0.5):
    s = testsystems.water_ligand_23k()
    return dict(
        x=s.x, params=s.params, box=s.box, exclusion_idxs=s.exclusion_idxs, scales=s.scales,
        plane=s.lambda_plane_idxs, offset=s.lambda_offset_idxs, lam=lam, beta=s.beta, cutoff=s.cutoff,
        interpolated=False, water=True,
    )


def _case_random(n, seed, lam=0.1):
    rng = np.random.default_rng(seed)
    c = small_water_case(rng, n)
    c.update(lam=lam, beta=2.0, cutoff=1.0, interpolated=False, water=False)
    return c


def _case_golden(name):
    g = load_golden(name)
    return dict(
        x=g["x"], params=g["params"], box=g["box"], exclusion_idxs=g["exclusion_idxs"], scales=g["scales"],
        plane=g["lambda_plane_idxs"], offset=g["lambda_offset_idxs"], lam=g["lam"], beta=g["beta"],
        cutoff=g["cutoff"], interpolated=True, water=False,
    )


CASES = {
    "water3k": _case_water3k,
    "water23k_lam0.5": _case_water23k,
    "random33": lambda: _case_random(33, 1),
    "random231": lambda: _case_random(231, 2),
    "random1050": lambda: _case_random(1050, 3, lam=0.2),
    "golden_repro": lambda: _case_golden("repro"),
    "golden_bad_test_547": lambda: _case_golden("bad_test_547"),
}


def _nonbonded(c):
    cls = P.NonbondedInterpolated if c["interpolated"] else P.Nonbonded
    return cls(c["exclusion_idxs"], c["scales"], c["plane"], c["offset"], c["beta"], c["cutoff"])


def _ref(c):
    return refgpu.RefNonbonded(
        c["exclusion_idxs"], c["scales"], c["plane"], c["offset"], c["beta"], c["cutoff"], c["interpolated"]
    )


def _inputs(c):
    return f32_round(c["x"]), f32_round(c["params"]), np.asarray(c["box"], dtype=np.float64)


needs_ref = pytest.mark.skipif(not refgpu.available(), reason="reference CUDA build (oracle/_ref) not present")


@needs_ref
@pytest.mark.parametrize("name", list(CASES))
def test_bitexact_vs_reference_kernel(name):
    c = CASES[name]()
    x, p, box = _inputs(c)
    mine = _nonbonded(c).unbound_impl(np.float32)
    ref = _ref(c)
    combos = list(itertools.product([False, True], repeat=4)) if x.shape[0] <= 1050 else [
        (True, True, True, True),
        (True, False, False, False),
        (False, False, False, True),
        (True, False, True, False),
    ]
    for combo in combos:
        a = run_device(mine, x, p, box, c["lam"], *combo)
        b = run_device(ref, x, p, box, c["lam"], *combo, runner=ref_runner)
        for k, label in enumerate(["du_dx", "du_dp", "du_dl", "u"]):
            if a[k] is None:
                assert b[k] is None
                continue
            if not np.array_equal(a[k], b[k]):
                diff = np.flatnonzero(np.asarray(a[k]).ravel() != np.asarray(b[k]).ravel())
                pytest.fail(f"{name} {combo} {label}: {diff.size} of {np.size(a[k])} differ, first {diff[:5]}")


@pytest.mark.parametrize("name", list(CASES))
def test_tolerance_vs_fp64_oracle(name):
    c = CASES[name]()
    x, p, box = _inputs(c)
    mine = _nonbonded(c).unbound_impl(np.float32)
    du_dx, du_dp, du_dl, u = decode(run_device(mine, x, p, box, c["lam"]), p.shape)
    o = Oracle(c["plane"], c["offset"], c["beta"], c["cutoff"], c["exclusion_idxs"], c["scales"], c["interpolated"])
    r_dx, r_dp, r_dl, r_u = o(x, p, box, c["lam"])
    ef = force_error(r_dx, du_dx)
    eu = abs(u - r_u) / max(abs(r_u), 1.0)
    edp = rel_error(r_dp, du_dp)
    edl = abs(du_dl - r_dl) / max(abs(r_dl), 1.0)
    print(f"\n[{name}] force {ef:.2e} u {eu:.2e} du_dp {edp:.2e} du_dl {edl:.2e} (u={u:.6f} ref {r_u:.6f})")
    if refgpu.available():
        k_dx, k_dp, k_dl, k_u = decode(run_device(_ref(c), x, p, box, c["lam"], runner=ref_runner), p.shape)
        ref_ef = force_error(r_dx, k_dx)
        print(f"[{name}] reference kernel: force {ref_ef:.2e} u {abs(k_u - r_u) / max(abs(r_u), 1.0):.2e}")
        assert ef <= ref_ef * (1 + 1e-6) + 1e-12
    if c["water"]:
        assert ef <= TOL_FORCE_WATER
        assert eu <= TOL_ENERGY_WATER
        assert edp <= TOL_FORCE_WATER
        assert edl <= TOL_FORCE_WATER
    else:
        assert ef <= TOL_RANDOM
        assert eu <= TOL_RANDOM
        assert edp <= TOL_RANDOM
        assert edl <= TOL_RANDOM


@pytest.mark.parametrize("rows", [32, 16, 8])
@pytest.mark.parametrize("name", ["water23k_lam0.5", "golden_repro"])
def test_nblist_covers_every_pair_within_cutoff(name, rows):
    """Every pair within the list radius (cutoff + the 0.1 nm padding) sits in
    the tile list of the lower slot's row group (tests/test_nblist.py:70-94
    against brute force), for row groups of 32, 16 and 8 slots: pairs that
    start just outside the cutoff can come within it before the next rebuild."""
    from scipy.spatial import cKDTree

    c = CASES[name]()
    x, p, box = _inputs(c)
    impl = _nonbonded(c).unbound_impl(np.float32)
    impl.set_tile_rows(rows)
    impl.execute(x, p, box, c["lam"])
    perm, tiles, got_rows = impl.get_nblist()
    assert got_rows == rows
    assert np.array_equal(np.sort(perm), np.arange(perm.size))
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size, dtype=perm.dtype)
    L = np.diag(box)
    xw = x - L * np.floor(x / L)
    xw = np.minimum(xw, np.nextafter(L, 0))
    pairs = cKDTree(xw, boxsize=L).query_pairs(c["cutoff"] + 0.1 - 1e-4, output_type="ndarray")
    si, sj = inv[pairs[:, 0]], inv[pairs[:, 1]]
    lo, hi = np.minimum(si, sj), np.maximum(si, sj)
    sets = [set(t.tolist()) for t in tiles]
    missing = sum(1 for a, b in zip(lo.tolist(), hi.tolist()) if b not in sets[a // rows])
    assert missing == 0
    for t in tiles:
        assert len(t) == len(set(t.tolist()))


def test_all_selective_variants_agree_and_are_deterministic():
    """Every output is bitwise the same in all 16 variants and on repeated calls
    (tests/common.py:451-477)."""
    c = CASES["random231"]()
    x, p, box = _inputs(c)
    mine = _nonbonded(c).unbound_impl(np.float32)
    full = run_device(mine, x, p, box, c["lam"])
    for combo in itertools.product([False, True], repeat=4):
        for _rep in range(2):
            out = run_device(mine, x, p, box, c["lam"], *combo)
            for k in range(4):
                if combo[k]:
                    assert np.array_equal(out[k], full[k])
                else:
                    assert out[k] is None


def test_hilbert_sort_on_off_bitwise_golden_repro():
    """tests/test_nonbonded.py:322-342 (fma compiler bug regression)."""
    c = _case_golden("repro")
    x, p, box = c["x"], c["params"], c["box"]
    a_impl = _nonbonded(c).unbound_impl(np.float32)
    b_impl = _nonbonded(c).unbound_impl(np.float32)
    b_impl.disable_hilbert_sort()
    a = a_impl.execute(x, p, box, c["lam"])
    b = b_impl.execute(x, p, box, c["lam"])
    for k in range(4):
        np.testing.assert_array_equal(a[k], b[k])


@pytest.mark.parametrize("rows", [16, 8])
@pytest.mark.parametrize("name", ["water23k_lam0.5", "random1050", "golden_repro"])
def test_tile_rows_bitwise_equal(name, rows):
    """Neighbour-list tiles of 16 (the default) or 8 rows give the fixed-point
    outputs of 32-row tiles bit for bit (one window and several windows): du_dx and du_dp
    per atom; u and du_dl as sums, since a pair's u and du_dl go to the atom
    in the lower slot, and the slot order within a row group differs."""
    c = CASES[name]()
    x, p, box = _inputs(c)
    a_impl = _nonbonded(c).unbound_impl(np.float32)
    a_impl.set_tile_rows(32)
    b_impl = _nonbonded(c).unbound_impl(np.float32)
    b_impl.set_tile_rows(rows)

    def same(a, b, per_atom):
        if per_atom:
            np.testing.assert_array_equal(a, b)
        else:
            assert int(np.sum(a, dtype=np.uint64)) == int(np.sum(b, dtype=np.uint64))

    fa = a_impl._execute_fixed(x, p, box, c["lam"], True, True, True, True)
    fb = b_impl._execute_fixed(x, p, box, c["lam"], True, True, True, True)
    for k in range(4):
        same(fa[k], fb[k], k < 2)
    lams = np.linspace(0.0, 1.0, 5)
    wa = a_impl.execute_windows_fixed(x, p, box, lams)
    wb = b_impl.execute_windows_fixed(x, p, box, lams)
    for k in range(4):
        for w in range(lams.size):
            same(wa[k][w], wb[k][w], k < 2)


def test_golden_bad_test_547_du_dl_exactly_zero():
    """tests/test_nonbonded.py:303-320."""
    c = _case_golden("bad_test_547")
    impl = _nonbonded(c).unbound_impl(np.float32)
    du_dx, du_dp, du_dl, u = impl.execute(c["x"], c["params"], c["box"], c["lam"])
    assert du_dl == 0.0
    assert np.all(np.isfinite(du_dx)) and np.isfinite(u)


def test_nblist_rebuild_cadence_bitwise():
    """padding 0 (rebuild every call) vs 0.1: identical results (tests/test_nonbonded.py:103-158)."""
    c = _case_water3k()
    rng = np.random.default_rng(2021)
    x0 = c["x"]
    N = x0.shape[0]
    padding = 0.1
    deltas = (rng.random((N, 3)) - 0.5) / (0.5 * (2 * np.sqrt(3)) / padding)
    ref_impl = _nonbonded(c).unbound_impl(np.float32)
    ref_impl.set_nblist_padding(0.0)
    test_impl = _nonbonded(c).unbound_impl(np.float32)
    test_impl.set_nblist_padding(padding)
    for x in [x0, x0 + deltas]:
        a = ref_impl.execute(x, c["params"], c["box"], 0.0)
        b = test_impl.execute(x, c["params"], c["box"], 0.0)
        for k in range(4):
            np.testing.assert_array_equal(a[k], b[k])
    assert test_impl.nblist_stats()[2] == 1  # the small moves did not trigger a rebuild
    assert ref_impl.nblist_stats()[2] == 2


def test_box_resize_rebuilds():
    """tests/test_nonbonded.py:252-299: large box then the real box, both correct."""
    c = _case_random(231, 7, lam=0.1)
    x, p, box = _inputs(c)
    impl = _nonbonded(c).unbound_impl(np.float32)
    o = Oracle(c["plane"], c["offset"], c["beta"], c["cutoff"], c["exclusion_idxs"], c["scales"])
    for b in [box + np.eye(3) * 1000, box]:
        du_dx, _, _, u = impl.execute(x, p, b, c["lam"])
        r_dx, _, _, r_u = o(x, p, b, c["lam"])
        assert force_error(r_dx, du_dx) <= TOL_RANDOM
        assert abs(u - r_u) <= TOL_RANDOM * max(abs(r_u), 1)


def test_box_errors():
    """tests/test_nonbonded.py:442-497."""
    c = _case_random(33, 11)
    x, p, box = _inputs(c)
    impl = _nonbonded(c).unbound_impl(np.float32)
    impl.execute_selective(x, p, box, 0.0, True, True, True, True)
    db_cutoff = (c["cutoff"] + 0.1) * 2
    impl.execute_selective(x, p, np.eye(3) * db_cutoff, 0.0, True, True, True, True)
    with pytest.raises(RuntimeError, match="non-ortholinear box"):
        impl.execute_selective(x, p, np.ones((3, 3)) * db_cutoff**2, 0.0, True, True, True, True)
    with pytest.raises(RuntimeError, match="more than half"):
        impl.execute_selective(x, p, np.eye(3) * (db_cutoff * 0.3), 0.0, True, True, True, True)
    # the handle stays usable after an error
    impl.execute_selective(x, p, box, 0.0, True, True, True, True)


def test_argument_errors_on_execute():
    """tests/nonbonded/test_nonbonded_all_pairs.py:28-47."""
    pot = P.NonbondedAllPairs([0], [0], 2.0, 1.1).unbound_impl(np.float32)
    with pytest.raises(RuntimeError, match="expected N == N_, got N=2, N_=1"):
        pot.execute(np.zeros((2, 3)), np.zeros((1, 3)), np.eye(3) * 3, 0)
    with pytest.raises(RuntimeError, match=r"expected P == M\*N_\*3, got P=6, M\*N_\*3=3"):
        pot.execute(np.zeros((1, 3)), np.zeros((2, 3)), np.eye(3) * 3, 0)
    pot_i = P.NonbondedAllPairsInterpolated([0], [0], 2.0, 1.1).unbound_impl(np.float32)
    with pytest.raises(RuntimeError, match=r"expected P == M\*N_\*3, got P=3, M\*N_\*3=6"):
        pot_i.execute(np.zeros((1, 3)), np.zeros((1, 3)), np.eye(3) * 3, 0)


def test_fused_nonbonded_equals_separate_potentials_bitwise():
    """Nonbonded == AllPairs + PairListNegated (timemachine/lib/potentials.py:284-301;
    tests/nonbonded/test_consistency.py)."""
    c = _case_random(1050, 5, lam=0.3)
    x, p, box = _inputs(c)
    fused = _nonbonded(c).unbound_impl(np.float32)
    allp = P.NonbondedAllPairs(c["plane"], c["offset"], c["beta"], c["cutoff"]).unbound_impl(np.float32)
    excl = P.NonbondedPairListNegated(
        c["exclusion_idxs"], c["scales"], c["plane"], c["offset"], c["beta"], c["cutoff"]
    ).unbound_impl(np.float32)
    a = run_device(fused, x, p, box, c["lam"])
    b1 = run_device(allp, x, p, box, c["lam"])
    b2 = run_device(excl, x, p, box, c["lam"])
    with np.errstate(over="ignore"):
        for k in range(4):
            np.testing.assert_array_equal(a[k], b1[k] + b2[k])


def test_pair_list_vs_oracle_and_negation():
    c = _case_random(231, 9, lam=0.4)
    x, p, box = _inputs(c)
    pl = P.NonbondedPairList(c["exclusion_idxs"], c["scales"], c["plane"], c["offset"], c["beta"], c["cutoff"])
    pn = P.NonbondedPairListNegated(c["exclusion_idxs"], c["scales"], c["plane"], c["offset"], c["beta"], c["cutoff"])
    a = run_device(pl.unbound_impl(np.float32), x, p, box, c["lam"])
    b = run_device(pn.unbound_impl(np.float32), x, p, box, c["lam"])
    with np.errstate(over="ignore"):
        for k in range(4):
            np.testing.assert_array_equal(a[k], np.uint64(0) - b[k])
    du_dx, du_dp, du_dl, u = decode(a, p.shape)
    r = pair_list_oracle(x, p, box, c["lam"], c["plane"], c["offset"], c["beta"], c["cutoff"], c["exclusion_idxs"], c["scales"])
    assert force_error(r[0], du_dx) <= TOL_RANDOM
    assert abs(u - r[3]) <= TOL_RANDOM * max(1, abs(r[3]))


def test_all_pairs_subsets(rng):
    """Singleton subset -> zeros; improper subset (all atoms) -> bitwise equal
    (tests/nonbonded/test_nonbonded_all_pairs.py:75-128)."""
    N = 231
    conf = rng.uniform(0, 1, size=(N, 3))
    params = rng.uniform(0, 1, size=(N, 3))
    plane = rng.integers(-2, 3, size=N, dtype=np.int32)
    offset = rng.integers(-2, 3, size=N, dtype=np.int32)
    box = 3.0 * np.eye(3)
    for idx in rng.choice(N, size=3):
        pot = P.NonbondedAllPairs(plane, offset, 2.0, 1.1, np.array([idx], dtype=np.int32)).unbound_impl(np.float32)
        du_dx, du_dp, du_dl, u = pot.execute(conf, params, box, 0.1)
        assert (du_dx == 0).all() and (du_dp == 0).all() and du_dl == 0 and u == 0
    a = P.NonbondedAllPairs(plane, offset, 2.0, 1.1).unbound_impl(np.float32).execute(conf, params, box, 0.1)
    b = P.NonbondedAllPairs(plane, offset, 2.0, 1.1, np.arange(N, dtype=np.int32)).unbound_impl(np.float32).execute(
        conf, params, box, 0.1
    )
    for k in range(4):
        np.testing.assert_array_equal(a[k], b[k])


def test_all_pairs_subset_vs_oracle(rng):
    c = _case_random(231, 13, lam=0.2)
    x, p, box = _inputs(c)
    sub = np.sort(rng.choice(231, 101, replace=False)).astype(np.int32)
    pot = P.NonbondedAllPairs(c["plane"], c["offset"], c["beta"], c["cutoff"], sub).unbound_impl(np.float32)
    du_dx, du_dp, du_dl, u = pot.execute(x, p, box, c["lam"])
    o = Oracle(c["plane"], c["offset"], c["beta"], c["cutoff"], atom_idxs=sub)
    r = o(x, p, box, c["lam"])
    assert force_error(r[0], du_dx) <= TOL_RANDOM
    assert abs(u - r[3]) <= TOL_RANDOM * max(1, abs(r[3]))


def test_newton_third_law_exact_at_full_size():
    """Size-independent exact property at 22,840 atoms: every pair adds +v and -v
    in int64, so the du_dx column sums are exactly zero (mod 2^64)."""
    c = _case_water23k(0.5)
    x, p, box = _inputs(c)
    mine = _nonbonded(c).unbound_impl(np.float32)
    dx, dp, dl, u = run_device(mine, x, p, box, c["lam"])
    with np.errstate(over="ignore"):
        assert np.all(dx.sum(axis=0, dtype=np.uint64) == 0)
    again = run_device(mine, x, p, box, c["lam"])
    for k in range(4):
        assert np.array_equal(again[k], (dx, dp, dl, u)[k])


def test_execute_device_accumulates():
    """Outputs accumulate (+=) across calls; the caller zeroes them."""
    c = _case_random(231, 21)
    x, p, box = _inputs(c)
    impl = _nonbonded(c).unbound_impl(np.float32)
    once = run_device(impl, x, p, box, c["lam"])
    dx = torch.as_tensor(x, device="cuda")
    dp_ = torch.as_tensor(p, device="cuda").reshape(-1)
    db = torch.as_tensor(box, device="cuda")
    o = torch.zeros((x.shape[0], 3), dtype=torch.int64, device="cuda")
    impl.execute_device(dx, dp_, db, c["lam"], du_dx=o)
    impl.execute_device(dx, dp_, db, c["lam"], du_dx=o)
    torch.cuda.synchronize()
    with np.errstate(over="ignore"):
        np.testing.assert_array_equal(o.cpu().numpy().view(np.uint64), once[0] * np.uint64(2))


def test_bound_potential_and_batch():
    c = _case_random(231, 17)
    x, p, box = _inputs(c)
    nb = _nonbonded(c).bind(p)
    bp = nb.bound_impl(np.float32)
    du_dx, du_dl, u = bp.execute(x, box, c["lam"])
    ref = nb.unbound_impl(np.float32).execute(x, p, box, c["lam"])
    np.testing.assert_array_equal(du_dx, ref[0])
    assert u == ref[3] and du_dl == ref[2]
    fixed = bp.execute_fixed(x, box, c["lam"])
    assert fixed.dtype == np.uint64 and fixed.shape == (1,)
    lams = np.array([0.0, 0.5])
    xs = np.stack([x, x + 0.01])
    boxes = np.stack([box, box])
    res = nb.unbound_impl(np.float32).execute_selective_batch(xs, p[None], boxes, lams, True, True, True, True)
    assert res[0].shape == (2, 1, 2, x.shape[0], 3)
    single = nb.unbound_impl(np.float32).execute(xs[1], p, box, 0.5)
    np.testing.assert_array_equal(res[0][1, 0, 1], single[0])
    assert res[3][1, 0, 1] == single[3]
