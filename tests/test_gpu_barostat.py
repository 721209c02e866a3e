"""GPU tests that pin the MC barostat to the reference's rules.

1. Move by move against an FP64 host restatement of
   timemachine/cpp/src/barostat.cu:139-279 (proposal, centroid rescaling,
   Metropolis test with w = dU + P dV - N_groups kT ln(V'/V), step-size
   adaptation), given the move's two uniform draws; the energies before and
   after the move equal independent evaluations of the bound potentials.
2. The molecular ideal gas of tests/test_barostat.py:262-368: without
   intermolecular terms the mean volume is N_groups kT / P (rtol 1e-2).
3. Varying pressure (tests/test_barostat.py:196-259): a water box shrinks at
   1000 atm and grows back after set_pressure(1 atm) / set_interval(2).
"""

import numpy as np
import pytest

from timemachine_b200 import md
from timemachine_b200 import potentials as P
from timemachine_b200 import testsystems

pytestmark = pytest.mark.gpu

BOLTZ = 0.008314462618
AVOGADRO = 6.0221367e23
FX = 2.0**36


def _groups(s):
    return [np.flatnonzero(s.group_of == g) for g in range(s.group_of.max() + 1)]


def _v0(s, temperature, seed):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(s.N, 3)) * np.sqrt(BOLTZ * temperature / s.masses)[:, None]


def _bonded(s):
    return [
        P.HarmonicBond(s.bond_idxs).bind(s.bond_params).bound_impl(np.float32),
        P.HarmonicAngle(s.angle_idxs).bind(s.angle_params).bound_impl(np.float32),
    ]


def _all(s):
    nb = P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    return _bonded(s) + [nb.bind(s.params).bound_impl(np.float32)]


def _total_u_fixed(bps, x, box, lam):
    """Fixed-point total energy of the bound potentials (uint64, wrapping), as
    the barostat sums it."""
    total = np.zeros(1, dtype=np.uint64)
    for bp in bps:
        _, _, _, fu = bp.potential._execute_fixed(x, bp.params, box, lam, False, False, False, True)
        total += np.array([fu.sum(dtype=np.uint64)], dtype=np.uint64)
    return total[0]


def _fixed_value(a):
    """A fixed-point uint64 as the signed value it encodes."""
    return float(np.array([a], dtype=np.uint64).view(np.int64)[0]) / FX


def _fixed_diff(a, b):
    return float((np.array([a], dtype=np.uint64) - np.array([b], dtype=np.uint64)).view(np.int64)[0]) / FX


def _fixed_centroids(x, group_of, n_groups):
    """Group centroids through the int64 fixed-point sums of
    timemachine/cpp/src/barostat.cu:186-200 (llrint(x * 2^36), wrapping)."""
    fx = np.rint(x * FX).astype(np.int64).view(np.uint64)
    sums = np.zeros((n_groups, 3), dtype=np.uint64)
    for d in range(3):
        np.add.at(sums[:, d], group_of[group_of >= 0], fx[group_of >= 0, d])
    counts = np.bincount(group_of[group_of >= 0], minlength=n_groups).astype(np.float64)
    return sums.view(np.int64).astype(np.float64) / FX / counts[:, None]


def test_moves_follow_the_reference_rules():
    s = testsystems.build_system(903, 3.0, seed=11, n_ligand=8)
    lam, temperature, pressure_bar = 0.3, 300.0, 1.0
    bps = _all(s)
    # dt = 0: the integrator leaves x in place, so each call is one barostat move at x
    intg = md.LangevinIntegrator(temperature, 0.0, 1.0, s.masses, 5)
    groups = _groups(s)
    baro = md.MonteCarloBarostat(s.N, pressure_bar, temperature, groups, 1, 77)
    ctx = md.Context(s.x, _v0(s, temperature, 3), s.box, intg, bps, barostat=baro)
    n_groups = len(groups)
    kt = BOLTZ * temperature
    p_md = pressure_bar * AVOGADRO * 1e-25
    scale_host = None
    n_acc = n_att = 0
    accepted_total = 0
    for move in range(40):
        x0, box0 = ctx.get_x_t(), ctx.get_box()
        ctx.multiple_steps(np.array([lam]))
        m = ctx.barostat_last_move()
        x1, box1 = ctx.get_x_t(), ctx.get_box()
        V = box0[0, 0] * box0[1, 1] * box0[2, 2]
        if scale_host is None:
            scale_host = 0.01 * V
        assert m["pressure"] == p_md
        assert m["proposal_scale"] == scale_host
        assert 0.0 < m["rand0"] < 1.0 and 0.0 < m["rand1"] < 1.0
        dV = scale_host * 2 * (m["rand0"] - 0.5)
        assert m["volume_delta"] == dV
        length = np.cbrt((V + dV) / V)
        assert m["length_scale"] == pytest.approx(length, rel=1e-15, abs=0)
        # energy before the move: the bound potentials at (x0, box0), bit for bit
        assert m["u_before"] == _total_u_fixed(bps, x0, box0, lam)
        # trial coordinates: each group's centroid moved by the length scale about the box centre
        c = _fixed_centroids(x0, s.group_of, n_groups)
        centre = np.diag(box0) * 0.5
        x_trial = x0.copy()
        g = s.group_of
        x_trial[g >= 0] += ((c[g[g >= 0]] - centre) * m["length_scale"]) + centre - c[g[g >= 0]]
        box_trial = box0.copy()
        box_trial[np.diag_indices(3)] *= m["length_scale"]
        du = _fixed_diff(m["u_after"], m["u_before"])
        w = du + p_md * dV - n_groups * kt * np.log((V + dV) / V)
        accepted = not (w > 0 and m["rand1"] > np.exp(-w / kt))
        assert accepted == m["accepted"], (move, w)
        if accepted:
            np.testing.assert_array_equal(box1, box_trial)
            np.testing.assert_allclose(x1, x_trial, rtol=0, atol=1e-12)
            # the energy after the move: the bound potentials at the accepted trial state
            assert m["u_after"] == _total_u_fixed(bps, x1, box1, lam)
            accepted_total += 1
        else:
            np.testing.assert_array_equal(box1, box0)
            np.testing.assert_array_equal(x1, x0)
            u_host = _fixed_value(_total_u_fixed(bps, x_trial, box_trial, lam))
            assert _fixed_value(m["u_after"]) == pytest.approx(u_host, rel=1e-7, abs=1e-6)
        # step-size adaptation (barostat.cu:249-266)
        n_att += 1
        n_acc += int(accepted)
        if n_att >= 10:
            if n_acc < 0.25 * n_att:
                scale_host /= 1.1
                n_att = n_acc = 0
            elif n_acc > 0.75 * n_att:
                scale_host = min(scale_host * 1.1, V * 0.3)
                n_att = n_acc = 0
        assert m["volume_scale"] == pytest.approx(scale_host, rel=1e-15)
    assert 0 < accepted_total < 40
    acc, att, _ = ctx.barostat_stats()
    assert att == 40 and acc == accepted_total


def test_molecular_ideal_gas_volume():
    """Bonded terms only (no intermolecular energy): the mean volume of the
    second half of 10,000 steps (a move every 5) at 100 bar is
    N_groups kT / P within 1 % at 300, 600 and 1000 K."""
    s = testsystems.build_system(1000, 3.104, seed=21, n_ligand=0)
    groups = _groups(s)
    pressure_bar = 100.0
    p_md = pressure_bar * AVOGADRO * 1e-25
    interval, n_steps = 5, 10000
    actual, expected = [], []
    for T in [300.0, 600.0, 1000.0]:
        want = len(groups) * BOLTZ * T / p_md
        # start near the expected volume (2 % above), molecules moved with their centroids
        V0 = np.prod(np.diag(s.box))
        scale = (1.02 * want / V0) ** (1 / 3)
        c = np.array([s.x[g].mean(axis=0) for g in groups])
        centre = np.diag(s.box) * 0.5
        x = s.x.copy()
        for k, g in enumerate(groups):
            x[g] += (c[k] - centre) * scale + centre - c[k]
        box = s.box * scale
        intg = md.LangevinIntegrator(T, 1.5e-3, 1.0, s.masses, 2021)
        baro = md.MonteCarloBarostat(s.N, pressure_bar, T, groups, interval, 2021)
        ctx = md.Context(x, _v0(s, T, 9), box, intg, _bonded(s), barostat=baro)
        _, _, boxes = ctx.multiple_steps(np.zeros(n_steps), store_x_interval=interval)
        vols = np.prod(np.diagonal(boxes, axis1=1, axis2=2), axis=1)
        actual.append(vols[len(vols) // 2 :].mean())
        expected.append(want)
    print("\nideal gas volumes", actual, "expected", expected)
    np.testing.assert_allclose(actual, expected, rtol=1e-2)


def test_varying_pressure():
    """After relaxing at 1 atm, a water box shrinks at 1000 atm
    (set_pressure) and grows back at 1 atm with a new interval
    (set_pressure + set_interval), each mean volume at least 0.4 nm^3 apart
    (the reference test's margin; the expected shift is ~4 % of 30 nm^3)."""
    s = testsystems.build_system(1000, 3.104, seed=31, n_ligand=0)
    atm = 1.01325
    intg = md.LangevinIntegrator(300.0, 1.5e-3, 1.0, s.masses, 2021)
    baro = md.MonteCarloBarostat(s.N, 1.0 * atm, 300.0, _groups(s), 3, 2021)
    ctx = md.Context(s.x, _v0(s, 300.0, 4), s.box, intg, _all(s), barostat=baro)

    def mean_volume(n_steps, tail):
        _, _, boxes = ctx.multiple_steps(np.ones(n_steps), store_x_interval=10)
        v = np.prod(np.diagonal(boxes, axis1=1, axis2=2), axis=1)
        return v[-tail // 10 :].mean()

    v_eq = mean_volume(4000, 1500)
    baro.set_pressure(1000.0 * atm)
    v_high = mean_volume(3000, 1000)
    baro.set_pressure(1.0 * atm)
    baro.set_interval(2)
    assert baro.get_interval() == 2
    v_back = mean_volume(4000, 1500)
    print(f"\nV(1 atm) {v_eq:.3f} V(1000 atm) {v_high:.3f} V(1 atm again) {v_back:.3f}")
    assert v_high < v_eq - 0.4
    assert v_back > v_high + 0.4
