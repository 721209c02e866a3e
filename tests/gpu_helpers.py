"""GPU-side helpers: run the B200 potential (and the reference build) on device tensors."""

import numpy as np
import torch


def to_dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def run_device(impl, x, p, box, lam, du_dx=True, du_dp=True, du_dl=True, u=True, runner=None):
    """Execute through the C-ABI device entry; returns the raw uint64 outputs
    (du_dx [N,3], du_dp [P], sum du_dl, sum u) with None for skipped outputs."""
    N = x.shape[0]
    P = np.asarray(p).size
    dx = to_dev(x)
    dp_ = to_dev(p).reshape(-1)
    db = to_dev(box)
    o_dx = torch.zeros((N, 3), dtype=torch.int64, device="cuda") if du_dx else None
    o_dp = torch.zeros(P, dtype=torch.int64, device="cuda") if du_dp else None
    o_dl = torch.zeros(N, dtype=torch.int64, device="cuda") if du_dl else None
    o_u = torch.zeros(N, dtype=torch.int64, device="cuda") if u else None
    if runner is None:
        impl.execute_device(dx, dp_, db, lam, o_dx, o_dp, o_dl, o_u)
    else:
        runner(impl, dx, dp_, db, lam, o_dx, o_dp, o_dl, o_u)
    torch.cuda.synchronize()

    def host(t):
        return None if t is None else t.cpu().numpy().view(np.uint64)

    def total(t):
        return None if t is None else np.uint64(t.cpu().numpy().view(np.uint64).sum(dtype=np.uint64))

    return host(o_dx), host(o_dp), total(o_dl), total(o_u)


def ref_runner(ref, dx, dp_, db, lam, o_dx, o_dp, o_dl, o_u):
    ref.execute_device(dx, dp_, db, lam, o_dx, o_dp, o_dl, o_u, stream=torch.cuda.current_stream().cuda_stream)


def decode(out, params_shape):
    from timemachine_b200.fixed_point import du_dp_fixed_to_float, fixed_to_float

    dx, dp, dl, u = out
    return (
        None if dx is None else fixed_to_float(dx),
        None if dp is None else du_dp_fixed_to_float(dp).reshape(params_shape),
        None if dl is None else fixed_to_float(dl),
        None if u is None else fixed_to_float(u),
    )
