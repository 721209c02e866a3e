"""GPU tests of the MD drivers (Langevin integrator, MC barostat, Context) on
the nonbonded potential: graph replay equals eager launches bit for bit, one
step follows the reference's BAOAB update, the barostat moves the box."""

import numpy as np
import pytest

from timemachine_b200 import md
from timemachine_b200 import potentials as P
from timemachine_b200 import testsystems

pytestmark = pytest.mark.gpu

BOLTZ = 0.008314462618


def _bound_potentials(s):
    nb = P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    hb = P.HarmonicBond(s.bond_idxs)
    ha = P.HarmonicAngle(s.angle_idxs)
    return [
        hb.bind(s.bond_params).bound_impl(np.float32),
        ha.bind(s.angle_params).bound_impl(np.float32),
        nb.bind(s.params).bound_impl(np.float32),
    ]


def _v0(s, temperature, seed):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(s.N, 3)) * np.sqrt(BOLTZ * temperature / s.masses)[:, None]


def _context(s, use_graphs, dt=1.5e-3, temperature=300.0, seed=2024, barostat_interval=0):
    bps = _bound_potentials(s)
    intg = md.LangevinIntegrator(temperature, dt, 1.0, s.masses, seed)
    baro = None
    if barostat_interval:
        groups = [np.flatnonzero(s.group_of == g) for g in range(s.group_of.max() + 1)]
        baro = md.MonteCarloBarostat(s.N, 1.0, temperature, groups, barostat_interval, seed + 1)
    ctx = md.Context(s.x, _v0(s, temperature, seed), s.box, intg, bps, barostat=baro, use_graphs=use_graphs)
    return ctx, bps


def test_configs0_workload_runs_and_stays_finite():
    """1,000 waters: one evaluation, then 100 Langevin steps at 1.5 fs, 300 K, 1/ps."""
    s = testsystems.water_box_3k()
    ctx, bps = _context(s, True)
    du_dx, du_dl, u = bps[2].execute(s.x, s.box, 0.0)
    assert np.all(np.isfinite(du_dx)) and np.isfinite(u)
    ctx.multiple_steps(np.zeros(100))
    x = ctx.get_x_t()
    assert np.all(np.isfinite(x))
    assert np.max(np.linalg.norm(x - s.x, axis=1)) < 0.5
    v = ctx.get_v_t()
    T = np.sum(s.masses[:, None] * v * v) / (3 * s.N * BOLTZ)
    # the lattice start (random orientations) relaxes and heats the box; the
    # thermostat keeps it bounded
    assert 150 < T < 2000, T


def test_graph_replay_equals_eager_bitwise():
    """Integer forces + counter-based noise: the CUDA-graph path and the eager
    launch path give bitwise-identical trajectories (barostat included)."""
    s = testsystems.build_system(500, 2.9, seed=5, n_ligand=10)
    a, _ = _context(s, True, barostat_interval=5)
    b, _ = _context(s, False, barostat_interval=5)
    lam = np.full(40, 0.25)
    da, _, _ = a.multiple_steps(lam, store_du_dl_interval=10)
    db, _, _ = b.multiple_steps(lam, store_du_dl_interval=10)
    np.testing.assert_array_equal(a.get_x_t(), b.get_x_t())
    np.testing.assert_array_equal(a.get_v_t(), b.get_v_t())
    np.testing.assert_array_equal(a.get_box(), b.get_box())
    np.testing.assert_array_equal(da, db)
    assert da.shape == (4,)


@pytest.mark.parametrize("n_waters,edge,dt", [(500, 2.9, 2.0e-3), (3000, 4.48, 0.5e-3)])
def test_rebuild_cadence_graph_and_eager_agree(n_waters, edge, dt):
    """Graph-replayed and eager steps give the same trajectory, du_dl and
    number of rebuilds, with several rebuilds and steps without one in
    between; captured steps also record the potentials on parallel branches.
    The larger box takes the tile build's shifted-image test, the smaller one
    its per-pair wrapped test."""
    s = testsystems.build_system(n_waters, edge, seed=7, n_ligand=10)
    lam = np.full(120, 0.3)
    runs = []
    for use_graphs in (True, False):
        ctx, bps = _context(s, use_graphs, dt=dt, barostat_interval=25)
        dl, _, _ = ctx.multiple_steps(lam, store_du_dl_interval=20)
        rebuilds = bps[2].potential.nblist_stats()[2]
        runs.append((ctx.get_x_t(), ctx.get_v_t(), ctx.get_box(), dl, rebuilds))
    ref = runs[0]
    # several rebuilds, and steps without one in between
    assert 2 < ref[4] < len(lam), ref[4]
    for r in runs[1:]:
        for a, b in zip(ref[:4], r[:4]):
            np.testing.assert_array_equal(a, b)
        assert r[4] == ref[4]


def test_multi_step_graphs_with_frames_equal_eager():
    """Graph replay runs the steps between frames, du_dl samples and barostat
    moves as one captured graph per run (intervals 10, 7 and 25 do not line
    up); the frames, du_dl samples and final state equal eager steps bit for
    bit."""
    s = testsystems.build_system(500, 2.9, seed=13, n_ligand=10)
    lam = np.full(100, 0.4)
    runs = []
    for use_graphs in (True, False):
        ctx, _ = _context(s, use_graphs, dt=2.0e-3, barostat_interval=25)
        dl, xs, boxes = ctx.multiple_steps(lam, store_du_dl_interval=7, store_x_interval=10)
        runs.append((dl, xs, boxes, ctx.get_x_t(), ctx.get_v_t(), ctx.get_box()))
    assert runs[0][1].shape == (10, s.N, 3)
    for a, b in zip(runs[0], runs[1]):
        np.testing.assert_array_equal(a, b)


def test_fused_graph_steps_leave_the_potential_clean():
    """Captured multi-step runs hand the nonbonded potential's coordinate
    staging and force scatter to the integrator kernel. With the nonbonded
    potential first in the list (recorded on the capture stream, not on a
    forked branch) the trajectory equals eager steps bit for bit, and
    afterwards the same potential evaluates exactly like a fresh instance (no
    forces left in its accumulators, staging and work counter in order)."""
    s = testsystems.build_system(500, 2.9, seed=17, n_ligand=10)
    lam = np.full(60, 0.2)  # captured runs of 25, 25 and 10 steps
    runs = []
    for use_graphs in (True, False):
        bps = _bound_potentials(s)[::-1]
        intg = md.LangevinIntegrator(300.0, 2.0e-3, 1.0, s.masses, 31)
        ctx = md.Context(s.x, _v0(s, 300.0, 31), s.box, intg, bps, use_graphs=use_graphs)
        ctx.multiple_steps(lam)
        x, box = ctx.get_x_t(), ctx.get_box()
        runs.append((x, ctx.get_v_t(), bps[0].execute(x, box, 0.2)))
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    np.testing.assert_array_equal(runs[0][1], runs[1][1])
    fresh = _bound_potentials(s)[2].execute(runs[0][0], s.box, 0.2)
    for out in (runs[0][2], runs[1][2]):
        for a, b in zip(out, fresh):
            np.testing.assert_array_equal(a, b)


def test_single_step_follows_baoab_update():
    """Zero temperature (no noise): x1, v1 equal the BAOAB update of
    timemachine/cpp/src/integrator.cu:37-69 with the potential's forces."""
    s = testsystems.water_box_3k()
    dt = 1.0e-3
    bps = _bound_potentials(s)
    intg = md.LangevinIntegrator(0.0, dt, 1.0, s.masses, 1)
    v0 = _v0(s, 300.0, 3)
    ctx = md.Context(s.x, v0, s.box, intg, bps)
    ctx.multiple_steps(np.zeros(1))
    du_dx = sum(bp.execute(s.x, s.box, 0.0)[0] for bp in bps)
    v_mid = v0 + intg.cbs[:, None] * du_dx
    v1 = intg.ca * v_mid
    x1 = s.x + 0.5 * dt * (v_mid + v1)
    np.testing.assert_allclose(ctx.get_v_t(), v1, rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(ctx.get_x_t(), x1, rtol=0, atol=1e-12)


def test_barostat_attempts_and_accepts_moves():
    s = testsystems.build_system(1000, 3.104, seed=11)
    ctx, _ = _context(s, True, barostat_interval=5)
    ctx.multiple_steps(np.zeros(200))
    accepted, attempted, vscale = ctx.barostat_stats()
    assert attempted == 40
    assert 0 < accepted <= 40
    box = ctx.get_box()
    assert box[0, 0] == box[1, 1] == box[2, 2]
    assert box[0, 0] != s.box[0, 0]
    assert np.all(np.isfinite(ctx.get_x_t()))


def test_lambda_schedule_and_du_dl_recording():
    s = testsystems.build_system(500, 2.9, seed=9, n_ligand=12)
    ctx, _ = _context(s, True)
    lam = np.linspace(0.0, 0.5, 20)
    du_dl, xs, boxes = ctx.multiple_steps(lam, store_du_dl_interval=5, store_x_interval=10)
    assert du_dl.shape == (4,) and np.all(np.isfinite(du_dl))
    assert xs.shape == (2, s.N, 3) and boxes.shape == (2, 3, 3)
    np.testing.assert_array_equal(xs[-1], ctx.get_x_t())


def test_multiple_steps_U_matches_independent_evaluations():
    """Context.multiple_steps_U (timemachine/cpp/src/context.cu:139-234): the
    trajectory equals multiple_steps at the same lambda, and U[f, k] equals the
    summed fixed-point energies of the bound potentials at frame f, window k."""
    s = testsystems.build_system(500, 2.9, seed=9, n_ligand=12)
    a, bps = _context(s, True, barostat_interval=5)
    b, _ = _context(s, True, barostat_interval=5)
    windows = np.array([0.0, 0.1, 0.35, 0.5, 0.8, 1.0])
    U, xs, boxes = a.multiple_steps_U(0.35, 20, windows, 10, 10)
    assert U.shape == (2, windows.size) and xs.shape == (2, s.N, 3) and boxes.shape == (2, 3, 3)
    _, xs_b, _ = b.multiple_steps(np.full(20, 0.35), store_x_interval=10)
    np.testing.assert_array_equal(xs, xs_b)
    for f in range(2):
        for k, lam in enumerate(windows):
            total = sum(int(bp.execute_fixed(xs[f], boxes[f], lam)[0]) for bp in bps) % (1 << 64)
            signed = total - (1 << 64) if total >= (1 << 63) else total
            assert U[f, k] == np.float64(signed) / 2.0**36, (f, k)
    # 40 windows: two multi-window evaluations per stored frame
    U40, _, _ = a.multiple_steps_U(0.0, 5, np.linspace(0.0, 1.0, 40), 5, 0)
    assert U40.shape == (1, 40) and np.all(np.isfinite(U40))
