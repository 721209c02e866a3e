"""GPU tests of NonbondedInteractionGroup (timemachine/cpp/src/nonbonded_interaction_group.cu;
tests/nonbonded/test_nonbonded_interaction_group.py is the reference's suite
this follows): validation messages, zero interactions, tolerance against the
FP64 oracle, bit-exactness against the reference build, the exact identity
U_all = U_rows + U_cols + U_group in fixed point, multi-window equality and
neighbour-list coverage."""

import numpy as np
import pytest

from oracle.nonbonded_oracle import Oracle, force_error, interaction_group_oracle, rel_error
from oracle.refgpu import refgpu
from tests.helpers import f32_round, small_water_case
from timemachine_b200 import potentials as P
from timemachine_b200 import testsystems

pytestmark = pytest.mark.gpu

# FP32 pair arithmetic against FP64: the reference suite's float32 tolerance
# for this potential (rtol 1e-4, atol 5e-4 on du_dx,
# tests/nonbonded/test_nonbonded_interaction_group.py:66), as a relative force error.
TOL_FORCE = 1e-4
TOL_ENERGY = 1e-5


def _group(rows, plane, offset, beta, cutoff, interpolated=False):
    cls = P.NonbondedInteractionGroupInterpolated if interpolated else P.NonbondedInteractionGroup
    return cls(rows, plane, offset, beta, cutoff).unbound_impl(np.float32)


def test_validation_messages():
    def make(rows, n):
        return _group(rows, np.zeros(n, np.int32), np.zeros(n, np.int32), 1.0, 1.0)

    with pytest.raises(RuntimeError, match="row_atom_idxs must be nonempty"):
        make([], 1)
    with pytest.raises(RuntimeError, match="atom indices must be unique"):
        make([1, 1], 3)
    with pytest.raises(RuntimeError, match="number of idxs must be less than N"):
        make([0, 1, 2], 3)
    with pytest.raises(RuntimeError, match="indices values must be less than N"):
        make([0, 5], 3)


def test_zero_interactions(rng):
    """Row atoms shifted by twice the cutoff: every output is exactly zero."""
    N, NR, cutoff = 33, 15, 1.1
    conf = rng.uniform(0, 1, size=(N, 3))
    rows = rng.choice(N, size=NR, replace=False).astype(np.int32)
    conf[rows, 0] += 2 * cutoff
    params = rng.uniform(0, 1, size=(N, 3))
    g = _group(rows, np.zeros(N, np.int32), np.zeros(N, np.int32), 2.0, cutoff)
    du_dx, du_dp, du_dl, u = g.execute(conf, params, 10.0 * np.eye(3), 0.1)
    assert np.all(du_dx == 0) and np.all(du_dp == 0) and du_dl == 0 and u == 0


@pytest.mark.parametrize("num_atoms,num_rows", [(33, 1), (33, 15), (231, 1), (231, 15), (1050, 40)])
@pytest.mark.parametrize("interpolated", [False, True])
def test_against_oracle(rng, num_atoms, num_rows, interpolated):
    c = small_water_case(rng, num_atoms)
    N = c["x"].shape[0]
    rows = rng.choice(N, size=num_rows, replace=False).astype(np.int32)
    params = c["params"]
    if interpolated:
        params = np.concatenate([params, params * rng.uniform(0.5, 1.5, size=params.shape)])
    g = _group(rows, c["plane"], c["offset"], 2.0, 1.1, interpolated)
    x, box = f32_round(c["x"]), c["box"]
    p = f32_round(params)
    for lam in ([0.0, 0.1, 0.9, 1.0] if interpolated else [0.0, 0.1]):
        du_dx, du_dp, du_dl, u = g.execute(x, p, box, lam)
        rx, rp, rl, ru = interaction_group_oracle(
            x, p, box, lam, c["plane"], c["offset"], 2.0, 1.1, rows, interpolated
        )
        assert force_error(rx, du_dx) < TOL_FORCE, lam
        assert abs(u - ru) <= TOL_ENERGY * max(1.0, abs(ru)), (u, ru)
        assert abs(du_dl - rl) <= 1e-4 * max(1.0, abs(rl)), (du_dl, rl)
        assert rel_error(rp.reshape(-1), du_dp.reshape(-1), floor=1.0) < 1e-4


def test_fixed_point_identity_all_equals_rows_plus_cols_plus_group():
    """U_all = U_rows + U_cols + U_group and the same for du_dx, du_dp and du_dl,
    exactly in int64 fixed point: each pair is evaluated once with the same
    FP32 arithmetic by exactly one of the three right-hand potentials
    (the identity of tests/nonbonded/test_nonbonded_interaction_group.py:188-258)."""
    s = testsystems.build_system(900, 3.0, seed=33, n_ligand=30)
    rows = np.flatnonzero(s.lambda_offset_idxs != 0).astype(np.int32)
    cols = np.setdiff1d(np.arange(s.N), rows).astype(np.int32)
    args = (s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    allp = P.NonbondedAllPairs(*args).unbound_impl(np.float32)
    rowp = P.NonbondedAllPairs(*args, rows).unbound_impl(np.float32)
    colp = P.NonbondedAllPairs(*args, cols).unbound_impl(np.float32)
    grp = _group(rows, *args)
    for lam in [0.0, 0.35, 1.0]:
        outs = [pot._execute_fixed(s.x, s.params, s.box, lam, True, True, True, True) for pot in (allp, rowp, colp, grp)]
        for c, name in enumerate(["du_dx", "du_dp", "du_dl", "u"]):
            a, r, cc, g = (o[c] for o in outs)
            if c >= 2:
                a, r, cc, g = (v.sum(dtype=np.uint64) for v in (a, r, cc, g))
            # uint64 sums wrap modulo 2^64, as the fixed-point accumulators do
            total = np.add(np.add(r, cc, dtype=np.uint64), g, dtype=np.uint64)
            np.testing.assert_array_equal(a, total, err_msg=f"{name} lambda={lam}")


def test_multi_window_equals_single_window():
    s = testsystems.build_system(700, 3.0, seed=21, n_ligand=24)
    rows = np.flatnonzero(s.lambda_offset_idxs != 0).astype(np.int32)
    g = _group(rows, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    lams = np.linspace(0.0, 1.0, 9)
    multi = g.execute_windows_fixed(s.x, s.params, s.box, lams)
    for k, lam in enumerate(lams):
        single = g._execute_fixed(s.x, s.params, s.box, lam, True, True, True, True)
        for c in range(4):
            np.testing.assert_array_equal(multi[c][k], single[c])


def test_neighbour_list_covers_every_row_column_pair():
    s = testsystems.build_system(900, 3.0, seed=8, n_ligand=30)
    rows = np.flatnonzero(s.lambda_offset_idxs != 0).astype(np.int32)
    g = _group(rows, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    g.execute(s.x, s.params, s.box, 0.0)
    perm, tiles, R = g.get_nblist()
    NR = rows.size
    assert sorted(perm[:NR].tolist()) == sorted(rows.tolist())
    listed = set()
    for rb, cols in enumerate(tiles):
        assert np.all(cols >= NR)
        for r in range(rb * R, min(NR, rb * R + R)):
            for cs in cols:
                listed.add((int(perm[r]), int(perm[cs])))
    o = Oracle(s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    in_rows = np.zeros(s.N, bool)
    in_rows[rows] = True
    for i, j in o.pairs(s.x, s.box):
        if in_rows[i] != in_rows[j]:
            a, b = (i, j) if in_rows[i] else (j, i)
            assert (a, b) in listed


@pytest.mark.skipif(not refgpu.available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("interpolated", [False, True])
def test_bitexact_against_reference_build(rng, interpolated):
    s = testsystems.water_ligand_23k()
    rows = np.flatnonzero(s.lambda_offset_idxs != 0).astype(np.int32)
    params = s.params
    if interpolated:
        params = np.concatenate([params, params * rng.uniform(0.8, 1.2, size=params.shape)])
    g = _group(rows, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff, interpolated)
    ref = refgpu.RefInteractionGroup(rows, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff, interpolated)
    for lam in [0.0, 0.5, 1.0]:
        mine = g._execute_fixed(s.x, params, s.box, lam, True, True, True, True)
        theirs = ref.execute_host_fixed(s.x, params, s.box, lam)
        np.testing.assert_array_equal(mine[0], theirs[0], err_msg=f"du_dx lambda={lam}")
        np.testing.assert_array_equal(mine[1], theirs[1].reshape(mine[1].shape), err_msg=f"du_dp lambda={lam}")
        assert mine[2].sum(dtype=np.uint64) == theirs[2].sum(dtype=np.uint64)
        assert mine[3].sum(dtype=np.uint64) == theirs[3].sum(dtype=np.uint64)
        # forces only: the packed two-rows-per-lane sweep, with the group's rows ending mid row group
        forces = g._execute_fixed(s.x, params, s.box, lam, True, False, False, False)
        np.testing.assert_array_equal(forces[0], theirs[0], err_msg=f"forces-only du_dx lambda={lam}")
