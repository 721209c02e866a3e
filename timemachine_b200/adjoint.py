"""Differentiable nonbonded forces: a torch.autograd.Function over the B200 kernels.

``nonbonded_forces(impl, params, w_offsets, x, box, lam)`` returns the
forces-as-gradient du_dx [N,3] and du_dl (scalar), both float64, computed by the
FP32 nonbonded kernels with int64 fixed-point accumulation. Its backward is
the hand-written adjoint kernel (timemachine_b200/csrc/nb_adjoint.cuh): the
vector-Jacobian product with respect to the per-atom parameters (charge,
sigma/2, sqrt(epsilon)) and the per-atom lambda offsets (w = cutoff * (plane +
offset * lambda), the offsets taken as continuous), recomputed pair by pair in
FP64 rather than stored. The reference obtains the same derivatives by
differentiating its jax potential twice (timemachine/potentials/nonbonded.py).
"""

import torch

FIXED_EXPONENT = float(0x1000000000)


class NonbondedForces(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params, w_offsets, impl, x, box, lam):
        N = x.shape[0]
        du_dx = torch.zeros((N, 3), dtype=torch.int64, device=x.device)
        du_dl = torch.zeros(N, dtype=torch.int64, device=x.device)
        p = params.detach().contiguous()
        impl.execute_device(x, p.reshape(-1), box, lam, du_dx=du_dx, du_dl=du_dl)
        f = du_dx.to(torch.float64) / FIXED_EXPONENT
        dl = du_dl.sum().to(torch.float64) / FIXED_EXPONENT  # wrapping int64 sum, then decode
        ctx.save_for_backward(p, x, box)
        ctx.impl = impl
        ctx.lam = float(lam)
        ctx.n_offsets = w_offsets.numel()
        return f, dl

    @staticmethod
    def backward(ctx, g_dx, g_dl):
        p, x, box = ctx.saved_tensors
        N = x.shape[0]
        g_dx = torch.zeros((N, 3), dtype=torch.float64, device=x.device) if g_dx is None else g_dx.contiguous()
        g_dl = 0.0 if g_dl is None else float(g_dl)
        grad_p = torch.zeros(p.numel(), dtype=torch.float64, device=x.device)
        grad_w = torch.zeros(N, dtype=torch.float64, device=x.device)
        ctx.impl.adjoint_device(x, p.reshape(-1), box, ctx.lam, g_dx.to(torch.float64), g_dl, grad_p, grad_w)
        return grad_p.view_as(p), grad_w.view(ctx.n_offsets), None, None, None, None


def nonbonded_forces(impl, params, w_offsets, x, box, lam):
    """(du_dx [N,3], du_dl) differentiable in params [N,3] and w_offsets [N].

    impl: an unbound Nonbonded / NonbondedAllPairs / NonbondedPairList
    implementation (not interpolated) whose lambda offsets equal w_offsets
    (the offsets enter the kernels as the integers given at construction;
    w_offsets carries their gradient). x [N,3], box [3,3]: float64 CUDA
    tensors; params: float64 CUDA tensor."""
    return NonbondedForces.apply(params, w_offsets, impl, x.contiguous(), box.contiguous(), lam)
