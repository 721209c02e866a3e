"""CPU tests of the FP64 oracle: pinned to the reference's golden fixtures and
to an independent dense transcription of the reference's jax nonbonded_v3."""

import numpy as np
import pytest
import torch
from scipy.special import erfc

from oracle.nonbonded_oracle import (
    Oracle,
    candidate_pairs,
    exclusion_masks,
    force_vjp_oracle,
    interaction_group_oracle,
    pair_list_oracle,
)
from tests.conftest import load_golden
from tests.helpers import f32_round, small_water_case


def dense_nonbonded_v3(conf, params, box, lamb, charge_rescale_mask, lj_rescale_mask, beta, cutoff, plane, offset):
    """Line-by-line numpy transcription of timemachine/potentials/nonbonded.py:133-264
    (energy only): dense N x N, masks, keep_mask, sum / 2."""
    N = conf.shape[0]
    w = cutoff * (plane + offset * lamb)
    conf = np.concatenate([conf, w[:, None]], axis=1)
    box4 = np.eye(4) * 1000
    box4[:3, :3] = box
    charges, sig, eps = params[:, 0], params[:, 1], params[:, 2]
    sig_ij = sig[None, :] + sig[:, None]
    eps_ij = eps[None, :] * eps[:, None]
    ri, rj = conf[None, :, :], conf[:, None, :]
    diff = ri - rj
    bd = np.diag(box4)
    diff = diff - bd * np.floor(diff / bd + 0.5)
    d2 = np.sum(diff**2, axis=-1)
    eye = np.eye(N, dtype=bool)
    d2 = np.where(eye, 0, d2)
    dij = np.where(eye, 0, np.sqrt(d2))
    keep = np.ones((N, N)) - np.eye(N)
    keep = np.where(eps_ij != 0, keep, 0)
    eps_ij = np.where(dij < cutoff, eps_ij, 0)
    sig_ij = np.where(keep, sig_ij, 0)
    eps_ij = np.where(keep, eps_ij, 0)
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = np.where(eye, 0, 1 / dij)
        sig2 = (sig_ij * inv) ** 2
        sig6 = sig2**3
        e_lj = np.where(keep, 4 * eps_ij * (sig6 - 1.0) * sig6, 0)
        qij = np.where(1 - np.eye(N), charges[None, :] * charges[:, None], 0)
        dd = np.where(1 - np.eye(N), dij, 0)
        e_q = np.where(1 - np.eye(N), qij * erfc(beta * dd) * inv, 0)
    e_q = np.where(dd > cutoff, 0, e_q)
    return np.sum((e_lj * lj_rescale_mask + e_q * charge_rescale_mask) / 2)


def rescale_masks(exclusion_idxs, scales, N):
    cm, lm = np.ones((N, N)), np.ones((N, N))
    for (i, j), (sc, sl) in zip(exclusion_idxs, scales):
        cm[i, j] = cm[j, i] = 1 - sc
        lm[i, j] = lm[j, i] = 1 - sl
    return cm, lm


@pytest.mark.parametrize("n_atoms", [33, 231])
@pytest.mark.parametrize("lamb", [0.0, 0.1, 0.7])
def test_oracle_matches_dense_transcription(rng, n_atoms, lamb):
    c = small_water_case(rng, n_atoms)
    o = Oracle(c["plane"], c["offset"], 2.0, 1.0, c["exclusion_idxs"], c["scales"])
    _, _, _, u = o(c["x"], c["params"], c["box"], lamb)
    cm, lm = rescale_masks(c["exclusion_idxs"], c["scales"], n_atoms)
    u_ref = dense_nonbonded_v3(c["x"], c["params"], c["box"], lamb, cm, lm, 2.0, 1.0, c["plane"], c["offset"])
    np.testing.assert_allclose(u, u_ref, rtol=1e-12, atol=1e-9)


def test_oracle_gradients_vs_finite_differences(rng):
    c = small_water_case(rng, 48, planes=(0, 2), offsets=(0, 2))
    o = Oracle(c["plane"], c["offset"], 2.0, 1.0, c["exclusion_idxs"], c["scales"])
    lamb = 0.3
    x, p, box = c["x"], c["params"], c["box"]
    pairs = o.pairs(x, box)  # fixed pair set so the FD stencil is smooth
    du_dx, du_dp, du_dl, _ = o(x, p, box, lamb, pairs=pairs)
    h = 1e-6

    def U(xx, pp, ll):
        return o(xx, pp, box, ll, pairs=pairs)[3]

    for k in rng.choice(x.size, 12, replace=False):
        xp, xm = x.copy(), x.copy()
        xp.flat[k] += h
        xm.flat[k] -= h
        fd = (U(xp, p, lamb) - U(xm, p, lamb)) / (2 * h)
        assert abs(fd - du_dx.flat[k]) <= 1e-5 * max(1.0, abs(fd))
    for k in rng.choice(p.size, 12, replace=False):
        pp_, pm = p.copy(), p.copy()
        pp_.flat[k] += h
        pm.flat[k] -= h
        fd = (U(x, pp_, lamb) - U(x, pm, lamb)) / (2 * h)
        assert abs(fd - du_dp.flat[k]) <= 1e-5 * max(1.0, abs(fd))
    fd = (U(x, p, lamb + h) - U(x, p, lamb - h)) / (2 * h)
    assert abs(fd - du_dl) <= 1e-5 * max(1.0, abs(fd))


def test_nonbonded_is_all_pairs_minus_scaled_exclusions(rng):
    """Nonbonded = AllPairs - PairList(exclusions, scales) (timemachine/lib/potentials.py:284-301)."""
    c = small_water_case(rng, 99)
    lamb = 0.2
    full = Oracle(c["plane"], c["offset"], 2.0, 1.0, c["exclusion_idxs"], c["scales"])
    allp = Oracle(c["plane"], c["offset"], 2.0, 1.0)
    a = full(c["x"], c["params"], c["box"], lamb)
    b = allp(c["x"], c["params"], c["box"], lamb)
    e = pair_list_oracle(
        c["x"], c["params"], c["box"], lamb, c["plane"], c["offset"], 2.0, 1.0, c["exclusion_idxs"], c["scales"]
    )
    for k in range(4):
        np.testing.assert_allclose(a[k], np.asarray(b[k]) - np.asarray(e[k]), rtol=1e-10, atol=1e-8)


def test_golden_bad_test_547_du_dl_is_zero():
    """tests/test_nonbonded.py:303-320: du_dl must be exactly zero for this input."""
    g = load_golden("bad_test_547")
    o = Oracle(
        g["lambda_plane_idxs"],
        g["lambda_offset_idxs"],
        g["beta"],
        g["cutoff"],
        g["exclusion_idxs"],
        g["scales"],
        interpolated=True,
    )
    _, du_dp, du_dl, u = o(g["x"], g["params"], g["box"], g["lam"])
    assert du_dl == 0.0
    assert np.isfinite(u) and du_dp.shape == g["params"].shape


def test_golden_repro_interpolated_endpoint():
    """repro.pkl.gz input at lambda=0 equals the plain potential on the lambda=0 parameters."""
    g = load_golden("repro")
    N = g["x"].shape[0]
    oi = Oracle(g["lambda_plane_idxs"], g["lambda_offset_idxs"], g["beta"], g["cutoff"], g["exclusion_idxs"], g["scales"], True)
    op = Oracle(g["lambda_plane_idxs"], g["lambda_offset_idxs"], g["beta"], g["cutoff"], g["exclusion_idxs"], g["scales"])
    pairs = oi.pairs(g["x"], g["box"])
    a = oi(g["x"], g["params"], g["box"], 0.0, pairs)
    b = op(g["x"], g["params"][:N], g["box"], 0.0, pairs)
    np.testing.assert_allclose(a[0], b[0], rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(a[3], b[3], rtol=1e-12)
    np.testing.assert_allclose(a[1][:N] + a[1][N:], b[1], rtol=1e-9, atol=1e-9)


def test_candidate_pairs_complete(rng):
    """The k-d tree candidate set equals brute force (tests/test_nblist.py:70-94 style)."""
    c = small_water_case(rng, 300)
    x, box, cutoff = c["x"], c["box"], 1.1
    pairs = candidate_pairs(x, box, cutoff)
    diag = np.diag(box)
    d = x[:, None, :] - x[None, :, :]
    d -= diag * np.round(d / diag)
    r = np.linalg.norm(d, axis=-1)
    iu = np.triu_indices(len(x), 1)
    ref = set(zip(iu[0][r[iu] < cutoff].tolist(), iu[1][r[iu] < cutoff].tolist()))
    got = set(map(tuple, pairs.tolist()))
    assert ref <= got
    # no far pairs beyond rounding
    for i, j in got - ref:
        assert r[i, j] < cutoff * (1 + 1e-8)


def test_exclusion_masks_lookup():
    pairs = np.array([[0, 1], [0, 2], [1, 2], [2, 5]])
    cm, lm = exclusion_masks(pairs, 6, np.array([[2, 1], [5, 2]]), np.array([[1.0, 0.5], [0.25, 0.0]]))
    np.testing.assert_array_equal(cm, [1, 1, 0, 0.75])
    np.testing.assert_array_equal(lm, [1, 1, 0.5, 1.0])


def test_oracle_f32_rounding_convention():
    a = np.array([0.1, 1 / 3])
    assert np.all(f32_round(a) == np.float32(a).astype(np.float64))


@pytest.mark.parametrize("interpolated", [False, True])
def test_interaction_group_oracle_is_all_minus_both_groups(rng, interpolated):
    """U_group = U_all - U_rows - U_cols (tests/nonbonded/test_nonbonded_interaction_group.py:188-258),
    with every derivative, in FP64."""
    c = small_water_case(rng, 180)
    N = c["x"].shape[0]
    rows = rng.choice(N, size=17, replace=False)
    cols = np.setdiff1d(np.arange(N), rows)
    params = c["params"]
    if interpolated:
        params = np.concatenate([params, params * 1.3])
    lam = 0.3
    g = interaction_group_oracle(c["x"], params, c["box"], lam, c["plane"], c["offset"], 2.0, 1.1, rows, interpolated)

    def allp(idxs):
        o = Oracle(c["plane"], c["offset"], 2.0, 1.1, interpolated=interpolated, atom_idxs=idxs)
        return o(c["x"], params, c["box"], lam)

    a, r, k = allp(None), allp(rows), allp(cols)
    for n in range(4):
        np.testing.assert_allclose(g[n], np.asarray(a[n]) - np.asarray(r[n]) - np.asarray(k[n]), rtol=1e-10, atol=1e-9)


def test_force_vjp_oracle_against_finite_differences(rng):
    """The double-backward reference of the adjoint against FP64 central
    differences (step 1e-4) of Phi = sum(G * du_dx) + g * du_dl."""
    c = small_water_case(rng, 90)
    N = c["x"].shape[0]
    G = rng.normal(size=(N, 3))
    g = 0.7
    lam = 0.4
    args = (c["box"], lam, c["plane"], c["offset"].astype(np.float64), 2.0, 1.1, c["exclusion_idxs"], c["scales"])
    pairs = candidate_pairs(c["x"], c["box"], 1.1)
    phi, gp, goff = force_vjp_oracle(c["x"], c["params"], *args, G, g, pairs=pairs)
    h = 1e-4
    for a, col in [(0, 0), (3, 1), (5, 2)]:
        pp, pm = c["params"].copy(), c["params"].copy()
        pp[a, col] += h
        pm[a, col] -= h
        fd = (force_vjp_oracle(c["x"], pp, *args, G, g, pairs=pairs)[0]
              - force_vjp_oracle(c["x"], pm, *args, G, g, pairs=pairs)[0]) / (2 * h)
        assert abs(fd - gp[a, col]) <= 1e-5 * max(1.0, abs(fd)), (a, col, fd, gp[a, col])
    for a in [1, 4]:
        op, om = c["offset"].astype(np.float64), c["offset"].astype(np.float64)
        op[a] += h
        om[a] -= h
        ap = (c["box"], lam, c["plane"], op, 2.0, 1.1, c["exclusion_idxs"], c["scales"])
        am = (c["box"], lam, c["plane"], om, 2.0, 1.1, c["exclusion_idxs"], c["scales"])
        fd = (force_vjp_oracle(c["x"], c["params"], *ap, G, g, pairs=pairs)[0]
              - force_vjp_oracle(c["x"], c["params"], *am, G, g, pairs=pairs)[0]) / (2 * h)
        assert abs(fd - goff[a]) <= 1e-5 * max(1.0, abs(fd)), (a, fd, goff[a])
