"""GPU tests of the adjoint kernel (timemachine_b200/csrc/nb_adjoint.cuh) and the
differentiable forces (timemachine_b200/adjoint.py): the vector-Jacobian
product of (du_dx, du_dl) with respect to parameters and lambda offsets
against the FP64 double-backward oracle and FP64 central finite differences,
for the Nonbonded potential (all pairs minus scaled exclusions)."""

import numpy as np
import pytest
import torch

from oracle.nonbonded_oracle import candidate_pairs, force_vjp_oracle
from tests.gpu_helpers import to_dev
from timemachine_b200 import potentials as P
from timemachine_b200 import testsystems
from timemachine_b200.adjoint import nonbonded_forces

pytestmark = pytest.mark.gpu

# The adjoint is FP64 on FP64 inputs, so it agrees with the FP64 oracle up to
# summation order; the end-to-end loss gradient also carries the FP32 forward
# (upstream gradients from FP32 forces), hence the looser bound there.
TOL_VJP = 1e-9
TOL_FD = 1e-5
TOL_LOSS_GRAD = 1e-3


def _system():
    s = testsystems.system_of_size(1200, seed=41, n_ligand=30)
    assert np.any(s.lambda_offset_idxs != 0)
    return s


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


def _adjoint(impl, s, lam, G, g):
    x, p, box = to_dev(s.x), to_dev(s.params).reshape(-1), to_dev(s.box)
    gp = torch.zeros(p.numel(), dtype=torch.float64, device="cuda")
    gw = torch.zeros(s.N, dtype=torch.float64, device="cuda")
    impl.adjoint_device(x, p, box, lam, to_dev(G), g, gp, gw)
    impl.check_device_error()
    torch.cuda.synchronize()
    return gp.cpu().numpy().reshape(-1, 3), gw.cpu().numpy()


@pytest.mark.parametrize("lam,rows", [(0.0, 32), (0.5, 32), (0.5, 16), (0.5, 8)])
def test_vjp_matches_double_backward_oracle(lam, rows):
    s = _system()
    impl = P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    impl = impl.unbound_impl(np.float32)
    impl.set_tile_rows(rows)
    rng = np.random.default_rng(3)
    G = rng.normal(size=(s.N, 3))
    g = 0.37
    gp, gw = _adjoint(impl, s, lam, G, g)
    _, rp, rw = force_vjp_oracle(
        s.x, s.params, s.box, lam, s.lambda_plane_idxs, s.lambda_offset_idxs.astype(np.float64), s.beta, s.cutoff,
        s.exclusion_idxs, s.scales, G, g,
    )
    print(f"[lambda={lam}, rows={rows}] relative error params {_rel(gp, rp):.2e} offsets {_rel(gw, rw):.2e}")
    assert _rel(gp, rp) < TOL_VJP
    assert _rel(gw, rw) < TOL_VJP or np.linalg.norm(rw) == 0
    # a second call gives the same gradient up to the order of the FP64 atomic sums
    gp2, _ = _adjoint(impl, s, lam, G, g)
    assert _rel(gp2, gp) < 1e-10


def test_vjp_on_a_list_built_by_a_multi_window_call():
    """A multi-window call builds its neighbour list with several tiles per work
    item, a single-window call with one; an adjoint that reuses a list built by
    either (no rebuild in between) walks it correctly."""
    s = _system()
    lam = 0.5
    impl = P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    impl = impl.unbound_impl(np.float32)
    rng = np.random.default_rng(6)
    G = rng.normal(size=(s.N, 3))
    g = 0.25
    impl.execute_windows_fixed(s.x, s.params, s.box, np.linspace(0.0, 1.0, 12))
    rebuilds = impl.nblist_stats()[2]
    gp, gw = _adjoint(impl, s, lam, G, g)
    assert impl.nblist_stats()[2] == rebuilds  # the adjoint reused the multi-window list
    _, rp, rw = force_vjp_oracle(
        s.x, s.params, s.box, lam, s.lambda_plane_idxs, s.lambda_offset_idxs.astype(np.float64), s.beta, s.cutoff,
        s.exclusion_idxs, s.scales, G, g,
    )
    assert _rel(gp, rp) < TOL_VJP
    assert _rel(gw, rw) < TOL_VJP


def test_vjp_matches_finite_differences():
    """FP64 central differences (step 1e-4) of Phi = sum(G * du_dx) + g * du_dl
    of the oracle, for ligand charges, sigmas, sqrt(eps) and offsets."""
    s = _system()
    lam = 0.5
    impl = P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    impl = impl.unbound_impl(np.float32)
    rng = np.random.default_rng(4)
    G = rng.normal(size=(s.N, 3))
    g = -0.8
    gp, gw = _adjoint(impl, s, lam, G, g)
    pairs = candidate_pairs(s.x, s.box, s.cutoff)
    lig = np.flatnonzero(s.lambda_offset_idxs != 0)
    off = s.lambda_offset_idxs.astype(np.float64)

    def phi(params, offsets):
        return force_vjp_oracle(
            s.x, params, s.box, lam, s.lambda_plane_idxs, offsets, s.beta, s.cutoff, s.exclusion_idxs, s.scales, G, g,
            pairs=pairs,
        )[0]

    h = 1e-4

    def crosses_cutoff(a, offsets):
        """Whether moving atom a's offset by +-h carries one of its pairs across
        the cutoff: the truncated potential (the reference's too) is
        discontinuous there, and a difference quotient across it measures the
        jump, not the derivative."""
        mine = pairs[(pairs[:, 0] == a) | (pairs[:, 1] == a)]
        i, j = mine[:, 0], mine[:, 1]
        L = np.diag(s.box)
        r = s.x[i] - s.x[j]
        r -= L * np.floor(r / L + 0.5)
        status = []
        for dh in (-h, h):
            o = offsets.copy()
            o[a] += dh
            w = s.cutoff * (s.lambda_plane_idxs + o * lam)
            d = np.sqrt((r * r).sum(1) + (w[i] - w[j]) ** 2)
            status.append(d < s.cutoff)
        return np.any(status[0] != status[1])

    errs, tested_offsets = [], 0
    for a in lig[:4]:
        for col in range(3):
            pp, pm = s.params.copy(), s.params.copy()
            pp[a, col] += h
            pm[a, col] -= h
            fd = (phi(pp, off) - phi(pm, off)) / (2 * h)
            errs.append(abs(fd - gp[a, col]) / max(1.0, abs(fd)))
    for a in lig:
        if tested_offsets == 4:
            break
        if crosses_cutoff(a, off):
            continue
        op, om = off.copy(), off.copy()
        op[a] += h
        om[a] -= h
        fd = (phi(s.params, op) - phi(s.params, om)) / (2 * h)
        errs.append(abs(fd - gw[a]) / max(1.0, abs(fd)))
        tested_offsets += 1
    assert tested_offsets == 4
    print(f"max relative error vs central differences: {max(errs):.2e}")
    assert max(errs) < TOL_FD


def test_autograd_function_loss_gradient():
    """Loss = mean squared force error + 0.1 du_dl^2 (the differentiation
    workload); gradients with respect to ligand parameters and offsets through
    torch.autograd against the FP64 oracle's."""
    s = _system()
    lam = 0.5
    impl = P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    impl = impl.unbound_impl(np.float32)
    rng = np.random.default_rng(5)
    target = rng.normal(size=(s.N, 3)) * 50.0
    x, box = to_dev(s.x), to_dev(s.box)
    params = to_dev(s.params).requires_grad_(True)
    w_off = to_dev(s.lambda_offset_idxs.astype(np.float64)).requires_grad_(True)
    du_dx, du_dl = nonbonded_forces(impl, params, w_off, x, box, lam)
    loss = ((du_dx - to_dev(target)) ** 2).mean() + 0.1 * du_dl**2
    loss.backward()
    # oracle: the same loss with FP64 forces
    from oracle.nonbonded_oracle import Oracle

    o = Oracle(s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff, s.exclusion_idxs, s.scales)
    fx, _, fl, _ = o(s.x, s.params, s.box, lam)
    G = 2.0 * (fx - target) / fx.size
    g = 0.2 * fl
    _, rp, rw = force_vjp_oracle(
        s.x, s.params, s.box, lam, s.lambda_plane_idxs, s.lambda_offset_idxs.astype(np.float64), s.beta, s.cutoff,
        s.exclusion_idxs, s.scales, G, g,
    )
    ep = _rel(params.grad.cpu().numpy(), rp)
    ew = _rel(w_off.grad.cpu().numpy(), rw)
    print(f"loss gradient relative error: params {ep:.2e} offsets {ew:.2e}")
    assert ep < TOL_LOSS_GRAD and ew < TOL_LOSS_GRAD


def test_unsupported_kinds_raise():
    s = _system()
    g = P.NonbondedInteractionGroup(
        np.flatnonzero(s.lambda_offset_idxs != 0), s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff
    ).unbound_impl(np.float32)
    with pytest.raises(RuntimeError, match="the adjoint covers"):
        _adjoint(g, s, 0.0, np.zeros((s.N, 3)), 0.0)
