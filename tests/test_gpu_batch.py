"""GPU tests of the replica batch (timemachine_b200/csrc/batch.cu): every
replica's outputs equal the single-system potentials' bit for bit, alone or in
any mix; MD of a replica equals the single-system Context bit for bit; graph
replay equals eager launches; schedule tuning changes no result."""

import numpy as np
import pytest

from timemachine_b200 import md
from timemachine_b200 import potentials as P
from timemachine_b200 import testsystems
from timemachine_b200.batch import ReplicaBatch

pytestmark = pytest.mark.gpu

MD = dict(temperature=300.0, dt=1.5e-3, friction=1.0)


def _systems():
    return [testsystems.system_of_size(n, seed=100 + k) for k, n in enumerate([600, 1500, 3100, 5200])]


def _single_fixed(s, lam, x=None):
    """Nonbonded + HarmonicBond + HarmonicAngle through the single-system path (raw fixed point)."""
    x = s.x if x is None else x
    nb = P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    nbi = nb.unbound_impl(np.float32)
    dx, dp, dl, u = nbi._execute_fixed(x, s.params, s.box, lam, True, True, True, True)
    for pot, params in [(P.HarmonicBond(s.bond_idxs), s.bond_params), (P.HarmonicAngle(s.angle_idxs), s.angle_params)]:
        bdx, _, _, bu = pot.unbound_impl(np.float32)._execute_fixed(x, params, s.box, lam, True, False, False, True)
        dx = dx + bdx
        u = u + bu
    return dx, dp, dl, u


def _v0(s, seed):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(s.N, 3)) * np.sqrt(md.BOLTZ * MD["temperature"] / s.masses)[:, None]


def test_every_replica_equals_single_system_evaluation():
    systems = _systems()
    lams = [0.0, 0.4, 1.0]
    b = ReplicaBatch()
    ids = {}
    for k, s in enumerate(systems):
        for lam in lams:
            ids[(k, lam)] = b.add(s, lam)
    b.evaluate()
    b.synchronize()
    for (k, lam), rid in ids.items():
        got = b.result_fixed(rid)
        want = _single_fixed(systems[k], lam)
        np.testing.assert_array_equal(got[0], want[0], err_msg=f"du_dx {k} {lam}")
        np.testing.assert_array_equal(got[1], want[1].reshape(-1, 3), err_msg=f"du_dp {k} {lam}")
        assert got[2].sum(dtype=np.uint64) == want[2].sum(dtype=np.uint64)
        assert got[3].sum(dtype=np.uint64) == want[3].sum(dtype=np.uint64)
        assert b.error(rid) == 0


def test_replica_alone_equals_replica_in_a_mix_and_membership_changes():
    systems = _systems()
    target = systems[1]
    alone = ReplicaBatch()
    a = alone.add(target, 0.3, v=_v0(target, 1), md=MD, seed=77)
    mix = ReplicaBatch()
    others = [mix.add(s, lam, v=_v0(s, 2), md=MD, seed=5) for s in systems for lam in (0.0, 1.0)]
    m = mix.add(target, 0.3, v=_v0(target, 1), md=MD, seed=77)
    # evaluation (per-atom u / du_dl are split by slot order, which may vary
    # within a Hilbert cell; their sums are the result)
    alone.evaluate()
    mix.evaluate()
    ra, rm = alone.result_fixed(a), mix.result_fixed(m)
    np.testing.assert_array_equal(ra[0], rm[0])
    np.testing.assert_array_equal(ra[1], rm[1])
    assert ra[2].sum(dtype=np.uint64) == rm[2].sum(dtype=np.uint64)
    assert ra[3].sum(dtype=np.uint64) == rm[3].sum(dtype=np.uint64)
    # MD, with replicas leaving and joining the mix between chunks
    alone.md(10, chunk=5)
    mix.md(10, chunk=5)
    mix.remove(others[0])
    mix.remove(others[3])
    extra = mix.add(systems[0], 0.5, v=_v0(systems[0], 3), md=MD, seed=9)
    alone.md(10, chunk=5)
    mix.md(10, chunk=5)
    np.testing.assert_array_equal(alone.get_x(a), mix.get_x(m))
    np.testing.assert_array_equal(alone.get_v(a), mix.get_v(m))
    assert np.all(np.isfinite(mix.get_x(extra)))


def test_replica_md_equals_single_system_context():
    """The Langevin step of the batch is the Context's (same Philox stream for
    the same seed, same forces): trajectories agree bit for bit."""
    s = _systems()[1]
    v0 = _v0(s, 4)
    lam = 0.2
    b = ReplicaBatch()
    rid = b.add(s, lam, v=v0, md=MD, seed=1234)
    b.md(30, chunk=10)
    intg = md.LangevinIntegrator(MD["temperature"], MD["dt"], MD["friction"], s.masses, 1234)
    nb = P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    bps = [
        P.HarmonicBond(s.bond_idxs).bind(s.bond_params).bound_impl(np.float32),
        P.HarmonicAngle(s.angle_idxs).bind(s.angle_params).bound_impl(np.float32),
        nb.bind(s.params).bound_impl(np.float32),
    ]
    ctx = md.Context(s.x, v0, s.box, intg, bps)
    ctx.multiple_steps(np.full(30, lam))
    np.testing.assert_array_equal(b.get_x(rid), ctx.get_x_t())
    np.testing.assert_array_equal(b.get_v(rid), ctx.get_v_t())


def test_graph_replay_equals_eager_and_tuning_changes_no_result():
    systems = _systems()[:3]
    runs = []
    for use_graph, tuning in [
        (True, None),
        (False, None),
        (True, dict(chunk=2, padding=0.06, grid_bits_offset=1)),
        (True, dict(chunk=1, rows=32)),
        (True, dict(chunk=4, rows=8)),
    ]:
        b = ReplicaBatch()
        if tuning:
            b.set_tuning(**tuning)
        ids = [b.add(s, lam, v=_v0(s, 6), md=MD, seed=11) for s in systems for lam in (0.1, 0.9)]
        b.md(24, chunk=8, use_graph=use_graph)
        b.evaluate()
        runs.append([(b.get_x(r), b.result_fixed(r)) for r in ids])
    for other in runs[1:]:
        for (x0, r0), (x1, r1) in zip(runs[0], other):
            np.testing.assert_array_equal(x0, x1)
            np.testing.assert_array_equal(r0[0], r1[0])
            np.testing.assert_array_equal(r0[1], r1[1])
            assert r0[2].sum(dtype=np.uint64) == r1[2].sum(dtype=np.uint64)
            assert r0[3].sum(dtype=np.uint64) == r1[3].sum(dtype=np.uint64)


def test_footprint_errors_and_autotune():
    s = testsystems.system_of_size(900, seed=3)
    b = ReplicaBatch()
    f_small = b.footprint(1000)
    f_big = b.footprint(20000)
    assert 0 < f_small < f_big
    rid = b.add(s, 0.0, md=MD, seed=1)
    assert b.bytes_in_use() >= b.footprint(s.N, len(s.exclusion_idxs), len(s.bond_idxs), len(s.angle_idxs))
    with pytest.raises(RuntimeError, match="unknown replica id"):
        b.error(rid + 100)
    # a box below twice cutoff + padding is reported for that replica only
    small = testsystems.system_of_size(300, seed=4, min_edge=2.0)
    bad = b.add(small, 0.0, md=MD, seed=2)
    b.evaluate()
    b.synchronize()
    assert b.error(bad) == 4
    assert b.error(rid) == 0
    b.remove(bad)
    best, timings = b.autotune(mode="eval", steps=2, repeats=1, candidates=[
        dict(chunk=2, padding=0.1, grid_bits_offset=0, pair_ctas_per_sm=0),
        dict(chunk=4, padding=0.1, grid_bits_offset=0, pair_ctas_per_sm=0),
    ])
    assert best in [t[0] for t in timings] and len(timings) == 2
    b.evaluate()
    want = _single_fixed(s, 0.0)
    got = b.result_fixed(rid)
    np.testing.assert_array_equal(got[0], want[0])
