"""FP64 CPU oracle of timemachine's nonbonded potential (TEST INFRASTRUCTURE).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use this
module, and only as the checker or the timed CPU baseline; the product never
imports it.

It restates the reference's jax implementation (jax is not installed here):

- timemachine/potentials/nonbonded.py:29-59 combining rules, Lennard-Jones and
  direct-space PME: sig_ij = sig_i + sig_j (sigma stored halved),
  eps_ij = eps_i * eps_j (sqrt(eps) stored), U_lj = 4 eps (s^12 - s^6),
  U_es = q_i q_j erfc(beta d) / d;
- :116-130 exclusions as rescale masks (mask = 1 - scale);
- :133-264 nonbonded_v3: 4D distances with w = cutoff*(plane + offset*lambda)
  (timemachine/potentials/jax_utils.py:32-67), minimum image
  d - box*floor(d/box + 0.5) (jax_utils.py:70-77) with an aperiodic 4th
  dimension, LJ kept where eps_ij != 0 and d < cutoff, electrostatics zeroed
  where d > cutoff, each pair counted once;
- :341-354 interpolated: p = (1 - lambda) p0 + lambda p1;
- lambda transforms (tests/test_parameter_interpolation.py:73-150, the
  reference's test of the four transform expressions): w uses f_w(lambda) and
  each parameter column its own f(lambda), p = (1 - f) p0 + f p1, with the
  transforms given here as torch functions of lambda.

Derivatives come from torch float64 autograd, as the reference tests take
jax.grad(argnums=(0, 1, 3)) (tests/common.py:448-450). Instead of the dense
N x N form, candidate pairs come from a periodic k-d tree on the 3D
coordinates (every pair within the 4D cutoff is within it in 3D), so the
oracle also runs at tens of thousands of atoms.

Parity status: pinned against the reference's golden fixtures
(tests/golden/) and against the reference CUDA kernel's outputs (see
tests/test_oracle.py and tests/test_gpu_parity.py).
"""

import numpy as np
import torch
from scipy.spatial import cKDTree


def candidate_pairs(x, box, cutoff, atom_idxs=None):
    """All pairs i < j whose 3D minimum-image distance is below cutoff (+ slack)."""
    x = np.asarray(x, dtype=np.float64)
    diag = np.diag(np.asarray(box, dtype=np.float64))
    sel = np.arange(x.shape[0]) if atom_idxs is None else np.asarray(atom_idxs)
    xs = x[sel] - diag * np.floor(x[sel] / diag)
    xs = np.minimum(xs, np.nextafter(diag, 0))  # boxsize is an open interval
    tree = cKDTree(xs, boxsize=diag)
    pairs = tree.query_pairs(cutoff * (1 + 1e-9) + 1e-12, output_type="ndarray")
    if pairs.size == 0:
        return np.zeros((0, 2), dtype=np.int64)
    pairs = sel[pairs]
    pairs = np.sort(pairs, axis=1)
    return pairs.astype(np.int64)


def exclusion_masks(pairs, N, exclusion_idxs, scales):
    """(charge_mask, lj_mask) per candidate pair: 1 - scale for listed pairs, else 1
    (timemachine/potentials/nonbonded.py:116-130)."""
    cm = np.ones(len(pairs))
    lm = np.ones(len(pairs))
    if exclusion_idxs is None or len(exclusion_idxs) == 0:
        return cm, lm
    e = np.sort(np.asarray(exclusion_idxs, dtype=np.int64).reshape(-1, 2), axis=1)
    s = np.asarray(scales, dtype=np.float64).reshape(-1, 2)
    ekey = e[:, 0] * N + e[:, 1]
    order = np.argsort(ekey)
    ekey, s = ekey[order], s[order]
    pkey = pairs[:, 0] * N + pairs[:, 1]
    pos = np.searchsorted(ekey, pkey)
    pos = np.minimum(pos, len(ekey) - 1)
    hit = ekey[pos] == pkey
    cm[hit] = 1 - s[pos[hit], 0]
    lm[hit] = 1 - s[pos[hit], 1]
    return cm, lm


def _identity(lam):
    return lam


def energy(x, params, box, lam, plane, offset, beta, cutoff, pairs, charge_mask, lj_mask, interpolated=False,
           transforms=None):
    """Total nonbonded energy (torch float64 scalar), differentiable in x, params, lam.

    transforms: None (identity) or (f_charge, f_sigma, f_epsilon, f_w), torch
    functions of lambda."""
    diag = torch.diagonal(box)
    N = x.shape[0]
    fq, fs, fe, fw = transforms if transforms is not None else (_identity,) * 4
    if interpolated:
        f = torch.stack([fq(lam), fs(lam), fe(lam)]).reshape(1, 3)
        params = (1 - f) * params[:N] + f * params[N:]
    w = cutoff * (plane + offset * fw(lam))
    i = torch.as_tensor(pairs[:, 0])
    j = torch.as_tensor(pairs[:, 1])
    dx = x[i] - x[j]
    dx = dx - diag * torch.floor(dx / diag + 0.5)
    dw = w[i] - w[j]
    d2 = (dx * dx).sum(-1) + dw * dw
    d = torch.sqrt(d2)
    q = params[:, 0]
    sig = params[:, 1]
    eps = params[:, 2]
    eps_ij = eps[i] * eps[j]
    sig_ij = sig[i] + sig[j]
    lj_keep = (eps_ij != 0) & (d < cutoff)
    es_keep = d <= cutoff
    # guard the masked-out lanes so their gradients are exactly zero
    d_lj = torch.where(lj_keep, d, torch.ones_like(d))
    s6 = (sig_ij / d_lj) ** 6
    u_lj = torch.where(lj_keep, 4 * eps_ij * (s6 - 1.0) * s6, torch.zeros_like(d))
    d_es = torch.where(es_keep, d, torch.ones_like(d))
    u_es = torch.where(es_keep, q[i] * q[j] * torch.special.erfc(beta * d_es) / d_es, torch.zeros_like(d))
    cm = torch.as_tensor(charge_mask)
    lm = torch.as_tensor(lj_mask)
    return (u_lj * lm + u_es * cm).sum()


class Oracle:
    """Reference semantics of Nonbonded / NonbondedAllPairs / NonbondedPairList(Negated)."""

    def __init__(
        self,
        lambda_plane_idxs,
        lambda_offset_idxs,
        beta,
        cutoff,
        exclusion_idxs=None,
        scales=None,
        interpolated=False,
        atom_idxs=None,
        transforms=None,
    ):
        self.plane = np.asarray(lambda_plane_idxs, dtype=np.float64)
        self.offset = np.asarray(lambda_offset_idxs, dtype=np.float64)
        self.beta = float(beta)
        self.cutoff = float(cutoff)
        self.exclusion_idxs = None if exclusion_idxs is None else np.asarray(exclusion_idxs)
        self.scales = None if scales is None else np.asarray(scales)
        self.interpolated = interpolated
        self.atom_idxs = atom_idxs
        self.transforms = transforms

    def pairs(self, x, box):
        return candidate_pairs(x, box, self.cutoff, self.atom_idxs)

    def __call__(self, x, params, box, lam, pairs=None):
        """(du_dx [N,3], du_dp [P/3,3], du_dl, u) in float64 numpy."""
        x = np.asarray(x, dtype=np.float64)
        N = x.shape[0]
        if pairs is None:
            pairs = self.pairs(x, box)
        cm, lm = exclusion_masks(pairs, N, self.exclusion_idxs, self.scales)
        tx = torch.tensor(x, dtype=torch.float64, requires_grad=True)
        tp = torch.tensor(np.asarray(params, dtype=np.float64), requires_grad=True)
        tl = torch.tensor(float(lam), dtype=torch.float64, requires_grad=True)
        tb = torch.tensor(np.asarray(box, dtype=np.float64))
        u = energy(
            tx,
            tp,
            tb,
            tl,
            torch.tensor(self.plane),
            torch.tensor(self.offset),
            self.beta,
            self.cutoff,
            pairs,
            cm,
            lm,
            self.interpolated,
            self.transforms,
        )
        gx, gp, gl = torch.autograd.grad(u, [tx, tp, tl], allow_unused=True)
        gl = 0.0 if gl is None else float(gl)
        return gx.numpy(), gp.numpy(), gl, float(u.detach())


def pair_list_oracle(x, params, box, lam, plane, offset, beta, cutoff, pair_idxs, scales, interpolated=False,
                     transforms=None):
    """Energy/derivatives of the listed pairs only, each scaled by (charge_scale, lj_scale)
    (tests/nonbonded/test_nonbonded_pair_list.py:35-47: nonbonded_v3_on_specific_pairs x scales)."""
    pair_idxs = np.asarray(pair_idxs, dtype=np.int64).reshape(-1, 2)
    scales = np.asarray(scales, dtype=np.float64).reshape(-1, 2)
    tx = torch.tensor(np.asarray(x, dtype=np.float64), requires_grad=True)
    tp = torch.tensor(np.asarray(params, dtype=np.float64), requires_grad=True)
    tl = torch.tensor(float(lam), dtype=torch.float64, requires_grad=True)
    tb = torch.tensor(np.asarray(box, dtype=np.float64))
    u = energy(
        tx,
        tp,
        tb,
        tl,
        torch.tensor(np.asarray(plane, dtype=np.float64)),
        torch.tensor(np.asarray(offset, dtype=np.float64)),
        float(beta),
        float(cutoff),
        pair_idxs,
        scales[:, 0],
        scales[:, 1],
        interpolated,
        transforms,
    )
    gx, gp, gl = torch.autograd.grad(u, [tx, tp, tl], allow_unused=True)
    gl = 0.0 if gl is None else float(gl)
    return gx.numpy(), gp.numpy(), gl, float(u.detach())


def interaction_group_oracle(x, params, box, lam, plane, offset, beta, cutoff, row_idxs, interpolated=False,
                             transforms=None):
    """Pairs (a, b) with a among row_idxs and b among the other atoms
    (timemachine/potentials/nonbonded.py:329-338, nonbonded_v3_interaction_groups
    over pairs_from_interaction_groups), unscaled."""
    x = np.asarray(x, dtype=np.float64)
    N = x.shape[0]
    rows = np.zeros(N, dtype=bool)
    rows[np.asarray(row_idxs, dtype=np.int64)] = True
    pairs = candidate_pairs(x, box, cutoff)
    pairs = pairs[rows[pairs[:, 0]] != rows[pairs[:, 1]]]
    ones = np.ones((len(pairs), 2))
    return pair_list_oracle(x, params, box, lam, plane, offset, beta, cutoff, pairs, ones, interpolated, transforms)


def force_vjp_oracle(x, params, box, lam, plane, offset, beta, cutoff, exclusion_idxs, scales, g_du_dx, g_du_dl,
                     pairs=None):
    """Reference for the adjoint kernel: with du_dx = dU/dx and du_dl = dU/dlambda
    of the Nonbonded energy (offsets taken as continuous), returns
    (Phi, dPhi/dparams [N,3], dPhi/doffsets [N]) for
    Phi = sum(g_du_dx * du_dx) + g_du_dl * du_dl, by FP64 double backward (the
    restatement of jax.grad applied twice to timemachine/potentials/nonbonded.py)."""
    x = np.asarray(x, dtype=np.float64)
    N = x.shape[0]
    if pairs is None:
        pairs = candidate_pairs(x, box, cutoff)
    cm, lm = exclusion_masks(pairs, N, exclusion_idxs, scales)
    tx = torch.tensor(x, requires_grad=True)
    tp = torch.tensor(np.asarray(params, dtype=np.float64), requires_grad=True)
    tl = torch.tensor(float(lam), dtype=torch.float64, requires_grad=True)
    toff = torch.tensor(np.asarray(offset, dtype=np.float64), requires_grad=True)
    tb = torch.tensor(np.asarray(box, dtype=np.float64))
    u = energy(tx, tp, tb, tl, torch.tensor(np.asarray(plane, dtype=np.float64)), toff, float(beta), float(cutoff),
               pairs, cm, lm)
    du_dx, du_dl = torch.autograd.grad(u, [tx, tl], create_graph=True)
    phi = (torch.as_tensor(np.asarray(g_du_dx, dtype=np.float64)) * du_dx).sum() + float(g_du_dl) * du_dl
    gp, goff = torch.autograd.grad(phi, [tp, toff], allow_unused=True)
    goff = torch.zeros(N, dtype=torch.float64) if goff is None else goff
    return float(phi.detach()), gp.numpy(), goff.numpy()


def force_error(ref, test):
    """max_i |F_ref - F_test|_inf / max(|F_ref,i|, 1) (tests/common.py:386-409 convention)."""
    ref = np.asarray(ref)
    test = np.asarray(test)
    norms = np.linalg.norm(ref, axis=-1, keepdims=True)
    norms = np.where(norms < 1.0, 1.0, norms)
    return float(np.max(np.abs((ref - test) / norms)))


def rel_error(ref, test, floor=1e-8):
    ref = np.asarray(ref, dtype=np.float64)
    test = np.asarray(test, dtype=np.float64)
    return float(np.max(np.abs(ref - test)) / max(np.max(np.abs(ref)), floor))
