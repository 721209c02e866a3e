#!/usr/bin/env python
"""Benchmark of the B200 nonbonded potential (one JSON line on rank 0).

Workload (one "step"): the 12 lambda windows (evenly spaced on [0, 1]) of the
22,840-atom water + ligand box (7,600 TIP3P-like waters + a 40-atom ligand
decoupled through w = 1.2 nm * lambda), each window one full nonbonded
evaluation (u, du_dx, du_dp, du_dl), all 12 through ONE multi-window call of
the C ABI (tmnb_potential_execute_windows_device) on device-resident inputs.
The same 12 windows as 12 single-window calls are reported beside it.
Synthetic, seeded inputs stand in for the reference's DHFR system (which
needs OpenMM to parametrise).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl tmnb|reference]

N > 1 (torchrun): every rank evaluates its own replica (replicas only, no
collective on the data path); value = all evaluations / max-over-ranks time.
The L2 cache is flushed (a 256 MiB write) before every timed step; only the
evaluations themselves are inside the CUDA events.

--impl reference: rank 0 times the reference's CPU implementation of the path
(the FP64 restatement of its jax nonbonded_v3 in oracle/, with all host
threads; jax itself is not installed) on one window per step, and, where the
reference CUDA build is present (oracle/_ref), the reference GPU kernel on the
same workload as an extra "reference_gpu" object.
"""

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

N_WINDOWS = 12
SEED = 2024

# FP32 operations of one in-cutoff pair of the full evaluation (u, du_dx,
# du_dp, du_dl), counted on the per-pair arithmetic of the pair kernel
# (timemachine_b200/csrc/nb_pair_math.cuh, pair_terms / sweep_tile in
# nb_kernels.cuh), which restates timemachine/cpp/src/kernels/nonbonded_common.cuh:38-140
# and k_nonbonded.cuh:424-512. FMA = 2; FMUL, FADD = 1; rsqrt, ex2 and the
# IEEE reciprocal = 1 each; the fixed-point scalings (v * 2^e) are counted,
# the float->int64 conversions and integer adds are not.
FLOP_TABLE = {
    "distance": {
        "3 coordinate differences": 3,
        "minimum image, 3 axes x (fmul by 1/L, 2 adds of the rounding constant, ffma)": 15,
        "d^2 = ffma(dz,dz,ffma(dx,dx,dy*dy))": 5,
    },
    "electrostatics": {
        "rsqrt": 1,
        "d = d2*inv_d, inv_d2 = inv_d^2": 2,
        "q_i q_j, (scale*q_i q_j)*inv_d": 3,
        "beta*d, -(beta d)^2, exp via ex2 (fmul + ex2)": 4,
        "1/(1 + 0.3275911 beta d): ffma + reciprocal": 3,
        "A&S 7.1.26 polynomial: 4 ffma": 8,
        "erfc = poly*t*e: 2 fmul": 2,
        "2/sqrt(pi)*beta*d, ffma(cbd, e, erfc), -inv_d2 * (...)": 4,
        "prefactor = qij_inv * factor": 1,
        "energy qij_inv * erfc": 1,
    },
    "forces": {"3 x (prefactor*delta)*2^36": 6},
    "charge derivatives": {"2 x (q_j*inv_d)*erfc": 4, "2 x fixed-point scaling": 2},
    "energy": {"fixed-point scaling": 1},
    "lennard_jones (both atoms carry epsilon)": {
        "eps_ij, sig_ij, s, s^2, s^4, s^6, s^6/d^2, s^5/d (2)": 9,
        "s^6 - 1": 1,
        "(scale*eps_ij)*s^6/d^2": 2,
        "ffma(s^6, 48, -24)": 2,
        "prefactor ffma": 2,
        "energy (3 fmul) + ffma": 5,
        "2 s^6 - 1 (ffma)": 2,
        "sigma gradient: 4 fmul": 4,
        "epsilon gradient: 3 fmul": 3,
        "2 x eps_grad*eps_j": 2,
        "3 fixed-point scalings": 3,
    },
    "lambda-dependent pair (an atom with a nonzero lambda offset)": {
        "dw, d^2 += dw^2 (fsub + ffma)": 3,
        "du_dl = ffma(dw*prefactor, dw_dl_i - dw_dl_j, .): fmul + fsub + ffma": 4,
        "fixed-point scaling": 1,
    },
}


def _table_sum(*groups):
    return sum(sum(FLOP_TABLE[g].values()) for g in groups)


# 65 per plain pair, +35 where both atoms carry LJ, +8 where either atom is lambda-dependent
FLOPS_PER_PAIR = _table_sum("distance", "electrostatics", "forces", "charge derivatives", "energy")
FLOPS_PER_LJ_PAIR = _table_sum("lennard_jones (both atoms carry epsilon)")
FLOPS_PER_ALCH_PAIR = _table_sum("lambda-dependent pair (an atom with a nonzero lambda offset)")
# DRAM bytes (read + write) of one 12-window pair-kernel launch on this
# workload, from an ncu capture of the same command (15.7 MB read, 0 written)
PAIR_LAUNCH_DRAM_BYTES = 15.7e6
# stages of a call timed by tmnb_potential_last_stage_ms
STAGE_PREPARE, STAGE_REBUILD, STAGE_PAIR, STAGE_FINALIZE = 0, 1, 2, 3


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="tmnb", choices=["tmnb", "reference"])
    ap.add_argument(
        "--profile",
        type=int,
        default=0,
        help="run only this many steps of the workload and exit; "
        "the command profiled by ncu for the committed kernel summaries",
    )
    ap.add_argument("--profile-outputs", default="all", choices=["all", "du_dx", "u"])
    ap.add_argument("--profile-precision", default="f32", choices=["f32", "f64"],
                    help="pair arithmetic of the windows/single profile modes")
    ap.add_argument(
        "--profile-mode",
        default="windows",
        choices=["windows", "single", "md", "batch", "batch_md", "grad"],
        help="windows: one 12-window call per step; single: one single-window call per step (cycling lambdas); "
        "md: Langevin steps of the MD workload (graph-replayed); batch: evaluations of 64 replicas (the first 8 "
        "systems of the batching mix x 8 windows); batch_md: batched Langevin steps of the same 64 replicas; grad: loss gradients of the differentiation workload on 4 frames",
    )
    ap.add_argument(
        "--forms",
        default="batch,serve,grad",
        help="comma-separated extra forms measured after the plain path: batch (512 replicas), serve (request "
        "loop), grad (adjoint loss gradients); '' for none",
    )
    return ap.parse_args()


def run_profile(args, local):
    import torch

    if args.profile_mode == "md":
        from timemachine_b200 import md
        from timemachine_b200 import potentials as P

        s = md_system()
        nb = P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
        bps = [
            P.HarmonicBond(s.bond_idxs).bind(s.bond_params).bound_impl(np.float32),
            P.HarmonicAngle(s.angle_idxs).bind(s.angle_params).bound_impl(np.float32),
            nb.bind(s.params).bound_impl(np.float32),
        ]
        baro = md.MonteCarloBarostat(s.N, 1.0, MD_TEMPERATURE, md_groups(s), MD_BARO_INTERVAL, SEED + 1)
        intg = md.LangevinIntegrator(MD_TEMPERATURE, MD_EQ_DT, 1.0, s.masses, SEED)
        ctx = md.Context(s.x, md_v0(s), s.box, intg, bps, baro)
        ctx.multiple_steps(np.full(args.profile, MD_LAMBDA))
        print(json.dumps({"profile_md_steps": args.profile}))
        return
    if args.profile_mode in ("batch", "batch_md"):
        from timemachine_b200.batch import ReplicaBatch

        systems, lambdas = batch_workload()
        b = ReplicaBatch()
        rng = np.random.default_rng(SEED + 5)
        for k, s in enumerate(systems[:8]):
            for w, lam in enumerate(lambdas):
                b.add(s, lam, v=_mb_velocities(rng, s, BATCH_MD["temperature"]), md=BATCH_MD, seed=1000 * k + w)
        for _ in range(args.profile):
            if args.profile_mode == "batch":
                b.evaluate()
            else:
                b.md(1, chunk=1, use_graph=False)
        b.synchronize()
        print(json.dumps({"profile_batch_" + ("evaluations" if args.profile_mode == "batch" else "md_steps"):
                          args.profile, "replicas": len(b)}))
        return
    if args.profile_mode == "grad":
        loss_and_grads = grad_workload(n_frames=4)[0]
        for _ in range(args.profile):
            loss_and_grads()
        torch.cuda.synchronize()
        print(json.dumps({"profile_loss_gradients": args.profile, "frames": 4}))
        return

    from timemachine_b200 import potentials as P

    s, x, p, lambdas = build_workload(0)
    impl = P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    impl = impl.unbound_impl(np.float64 if args.profile_precision == "f64" else np.float32)
    dev = torch.device("cuda", local)
    dx = torch.as_tensor(x, device=dev)
    dp = torch.as_tensor(p, device=dev).reshape(-1)
    db = torch.as_tensor(s.box, device=dev)
    N = s.N
    K = N_WINDOWS if args.profile_mode == "windows" else 1
    want = args.profile_outputs
    o_dx = torch.zeros((K, N, 3), dtype=torch.int64, device=dev) if want in ("all", "du_dx") else None
    o_dp = torch.zeros((K, p.size), dtype=torch.int64, device=dev) if want == "all" else None
    o_dl = torch.zeros((K, N), dtype=torch.int64, device=dev) if want == "all" else None
    o_u = torch.zeros((K, N), dtype=torch.int64, device=dev) if want in ("all", "u") else None
    for k in range(args.profile):
        if K > 1:
            impl.execute_windows_device(dx, dp, db, lambdas, o_dx, o_dp, o_dl, o_u)
        else:
            impl.execute_device(dx, dp, db, float(lambdas[k % N_WINDOWS]), o_dx, o_dp, o_dl, o_u)
    torch.cuda.synchronize()
    print(json.dumps({"profile_steps": args.profile, "mode": args.profile_mode, "outputs": want, "nblist": impl.nblist_stats()}))


def dist_setup():
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if torch.cuda.is_available():
        torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        # one process per GPU over NCCL; gloo where no GPU is present (the
        # CPU tests of the replica plumbing)
        backend = os.environ.get("TMNB_DIST_BACKEND", "nccl" if torch.cuda.is_available() else "gloo")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    QUERY = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"],
                stdout=open(self.path, "w"),
                stderr=subprocess.DEVNULL,
            )
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [c.strip() for c in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {
            "sm_mhz": float(np.median(sm)),
            "sm_max_mhz": float(max(smax)),
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def build_workload(rank):
    from timemachine_b200 import testsystems

    s = testsystems.water_ligand_23k(seed=SEED + rank)
    x = s.x.astype(np.float32).astype(np.float64)
    p = s.params.astype(np.float32).astype(np.float64)
    lambdas = np.linspace(0.0, 1.0, N_WINDOWS)
    return s, x, p, lambdas


def count_pairs(s, x, lambdas):
    """In-cutoff pairs (4D distance < cutoff) per window: (pairs, LJ pairs,
    lambda-dependent pairs), the excluded/scaled pairs included (the launch
    evaluates them too); plus the same counts over what one multi-window
    evaluation computes: pairs of two lambda-independent atoms once, the
    others once per window."""
    from scipy.spatial import cKDTree

    L = np.diag(s.box)
    xw = x - L * np.floor(x / L)
    xw = np.minimum(xw, np.nextafter(L, 0))
    pairs = cKDTree(xw, boxsize=L).query_pairs(s.cutoff, output_type="ndarray")
    i, j = pairs[:, 0], pairs[:, 1]
    d = x[i] - x[j]
    d -= L * np.round(d / L)
    d2 = (d * d).sum(1)
    excl = np.sort(np.asarray(s.exclusion_idxs).reshape(-1, 2), axis=1)
    # the scaled pairs are evaluated in the same launch: count them as pairs too
    ei, ej = excl[:, 0], excl[:, 1]
    de = x[ei] - x[ej]
    de -= L * np.round(de / L)
    i = np.concatenate([i, ei])
    j = np.concatenate([j, ej])
    d2 = np.concatenate([d2, (de * de).sum(1)])
    lj = (s.params[i, 2] != 0) & (s.params[j, 2] != 0)
    dep_atom = s.lambda_offset_idxs != 0
    dep = dep_atom[i] | dep_atom[j]
    out = []
    shared = [0, 0, 0]
    for k, lam in enumerate(lambdas):
        w = s.cutoff * (s.lambda_plane_idxs + s.lambda_offset_idxs * lam)
        keep = d2 + (w[i] - w[j]) ** 2 < s.cutoff**2
        out.append((int(keep.sum()), int((keep & lj).sum()), int((keep & dep).sum())))
        if k == 0:
            shared = [int((keep & ~dep).sum()), int((keep & ~dep & lj).sum()), 0]
        shared[0] += int((keep & dep).sum())
        shared[1] += int((keep & dep & lj).sum())
        shared[2] += int((keep & dep).sum())
    return out, len(excl), tuple(shared)


def flops_of(pairs, lj_pairs, dep_pairs):
    return pairs * FLOPS_PER_PAIR + lj_pairs * FLOPS_PER_LJ_PAIR + dep_pairs * FLOPS_PER_ALCH_PAIR


def measured_peaks():
    try:
        return json.load(open(os.path.join(HERE, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def stage_ms(lib, impl, stage):
    import ctypes

    from timemachine_b200 import _lib

    ms = ctypes.c_float()
    _lib.check(lib.tmnb_potential_last_stage_ms(impl.handle, stage, ctypes.byref(ms)))
    return ms.value


def hbm_roofline(N, K, ms, tiles, items, peak):
    """Achieved HBM GB/s of the bandwidth-bound stages of a K-window call,
    from their algorithmic bytes (the data each must move once) and their
    CUDA-event durations.

    prepare (k_check_prepare): reads x, the list's x, params (f64, 24 B each),
      plane + offset, slot order, lambda flag (13 B); writes K x 32 B of
      staged float4 coordinates + parameters and the flag.
    rebuild (sort, scatter, block bounds, tile build; on a rebuild call):
      reads x twice (keys, scatter) and params (LJ order); writes the slot
      order, the list's x, the staging (K x 32 B), bounds; the tiles
      (tiles x 32 column slots x 4 B) and work items (16 B).
    finalize (k_finalize + accumulator reset): reads the 8 accumulator arrays
      of the shared block and of the K window blocks (8 B each); adds K
      windows of outputs (du_dx, du_dp 24 B, du_dl, u 8 B: read + write);
      zeroes the blocks it read.
    """
    blocks = 1 + K if K > 1 else 1
    b_prepare = N * (24 + 24 + 24 + 13 + 1 + 32 * K)
    b_rebuild = N * (24 * 2 + 24 + 8 + 24 + 32 * K) + (N // 32 + 1) * 32 + tiles * 32 * 4 + items * 16
    b_finalize = N * (8 * 8 * blocks * 2 + K * 64 * 2)
    out = {}
    for name, b, t in [
        ("k_check_prepare", b_prepare, ms["prepare"]),
        ("rebuild_chain (k_bin_keys..k_build_tiles)", b_rebuild, ms["rebuild"]),
        ("k_finalize + reset", b_finalize, ms["finalize"]),
    ]:
        gbs = b / (t * 1e-3) / 1e9
        out[name] = {"bytes": int(b), "ms": t, "achieved_gbs": gbs, "frac": gbs / peak}
    return out


def output_errors(s, x, p, lam, fixed_by_precision):
    """Relative errors of (du_dx, du_dp, du_dl, u) against the FP64 oracle at
    one lambda window: forces by max_i |dF_i| / max(|F_i|, 1)
    (tests/common.py:386-409), du_dp by max |d| / max |ref|, u and du_dl by
    |d| / max(|ref|, 1)."""
    from oracle.nonbonded_oracle import Oracle, force_error, rel_error
    from timemachine_b200.fixed_point import du_dp_fixed_to_float, fixed_to_float, sum_fixed

    o = Oracle(s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff, s.exclusion_idxs, s.scales)
    r_dx, r_dp, r_dl, r_u = o(x, p, s.box, lam)
    res = {"lambda": float(lam), "oracle": "FP64 restatement of the reference's nonbonded_v3 (oracle/)"}
    for name, (fdx, fdp, fdl, fu) in fixed_by_precision.items():
        dx = fixed_to_float(fdx)
        dp = du_dp_fixed_to_float(fdp).reshape(p.shape)
        dl = fixed_to_float(sum_fixed(fdl))
        u = fixed_to_float(sum_fixed(fu))
        res[name] = {
            "du_dx": force_error(r_dx, dx),
            "du_dp": rel_error(r_dp, dp),
            "du_dl": abs(dl - r_dl) / max(abs(r_dl), 1.0),
            "u": abs(u - r_u) / max(abs(r_u), 1.0),
        }
    return res


def run_tmnb(args, world, rank, local):
    import ctypes

    import torch

    from timemachine_b200 import _lib
    from timemachine_b200 import potentials as P

    s, x, p, lambdas = build_workload(rank)
    N = s.N
    nb = P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    impl = nb.unbound_impl(np.float32)
    dev = torch.device("cuda", local)
    dx = torch.as_tensor(x, device=dev)
    dp = torch.as_tensor(p, device=dev).reshape(-1)
    db = torch.as_tensor(s.box, device=dev)
    K = N_WINDOWS
    o_dx = torch.zeros((K, N, 3), dtype=torch.int64, device=dev)
    o_dp = torch.zeros((K, p.size), dtype=torch.int64, device=dev)
    o_dl = torch.zeros((K, N), dtype=torch.int64, device=dev)
    o_u = torch.zeros((K, N), dtype=torch.int64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    lib = _lib.lib()

    def zero_outputs():
        o_dx.zero_()
        o_dp.zero_()
        o_dl.zero_()
        o_u.zero_()

    def one_step(pot=impl):
        zero_outputs()
        pot.execute_windows_device(dx, dp, db, lambdas, o_dx, o_dp, o_dl, o_u, stream=stream)

    # the single-window calls use their own potential, as a caller making only
    # single-window calls would (its neighbour list is built by one of them)
    impl1 = nb.unbound_impl(np.float32)

    def one_step_sequential():
        for k, lam in enumerate(lambdas):
            o_dx[k].zero_()
            o_dp[k].zero_()
            o_dl[k].zero_()
            o_u[k].zero_()
            impl1.execute_device(dx, dp, db, float(lam), o_dx[k], o_dp[k], o_dl[k], o_u[k], stream=stream)

    def timed(step_fn, steps=None):
        steps = args.steps if steps is None else steps
        for _ in range(args.warmup):
            step_fn()
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        barrier(world)
        torch.cuda.synchronize()
        for k in range(steps):
            flush.zero_()
            evs[k][0].record(stream)
            step_fn()
            evs[k][1].record(stream)
        torch.cuda.synchronize()
        barrier(world)
        return max_over_ranks(sum(a.elapsed_time(b) for a, b in evs), world)

    # timed region: K steps, L2 flushed before each, events around each step
    clk = ClockSampler(local).__enter__()  # sampled through the timed evaluations and the MD run
    total_ms = timed(one_step)
    tiles, items, rebuilds = impl.nblist_stats()
    seq_ms = timed(one_step_sequential)
    ms_per_step = total_ms / args.steps
    evals = args.steps * N_WINDOWS * world
    value = evals / (total_ms / 1e3)
    seq_value = evals / (seq_ms / 1e3)
    f32_fixed = [t[6].cpu().numpy().view(np.uint64) for t in (o_dx, o_dp, o_dl, o_u)]

    # per-stage durations of the multi-window call (events on the launching stream)
    _lib.check(lib.tmnb_potential_enable_timing(impl.handle, 1))
    st = {"prepare": [], "pair": [], "finalize": [], "rebuild": []}
    for _ in range(5):
        flush.zero_()
        one_step()
        for name, k in [("prepare", STAGE_PREPARE), ("pair", STAGE_PAIR), ("finalize", STAGE_FINALIZE)]:
            st[name].append(stage_ms(lib, impl, k))
    # rebuild calls: the coordinates alternate by 0.06 nm (> padding / 2), so every call rebuilds
    dx_shift = dx.clone()
    dx_shift[:, 0] += 0.06
    for k in range(6):
        flush.zero_()
        zero_outputs()
        impl.execute_windows_device(dx_shift if k % 2 == 0 else dx, dp, db, lambdas, o_dx, o_dp, o_dl, o_u,
                                    stream=stream)
        st["rebuild"].append(stage_ms(lib, impl, STAGE_REBUILD))
    _lib.check(lib.tmnb_potential_enable_timing(impl.handle, 0))
    pair_ms = st["pair"]
    _lib.check(lib.tmnb_potential_enable_timing(impl1.handle, 1))
    pair_ms_single = []
    for _ in range(2):
        for lam in lambdas:
            flush.zero_()
            impl1.execute_device(dx, dp, db, float(lam), o_dx[0], o_dp[0], o_dl[0], o_u[0], stream=stream)
            pair_ms_single.append(stage_ms(lib, impl1, STAGE_PAIR))
    _lib.check(lib.tmnb_potential_enable_timing(impl1.handle, 0))
    peak = ctypes.c_double()
    _lib.check(lib.tmnb_probe_fp32_peak(ctypes.byref(peak)))
    counts, n_excl, shared = count_pairs(s, x, lambdas)
    flops_launch = flops_of(*shared)
    pair_s = float(np.mean(pair_ms)) / 1e3
    achieved = flops_launch / pair_s / 1e12
    flops_single = float(np.mean([flops_of(*c) for c in counts]))
    achieved_single = flops_single / (float(np.mean(pair_ms_single)) / 1e3) / 1e12
    peaks = measured_peaks()
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    hbm = hbm_roofline(
        N, K, {k: float(np.median(v)) for k, v in st.items()}, tiles, items, hbm_peak
    )

    # FP64 pair arithmetic (unbound_impl(np.float64)): the same 12-window call
    impl64 = nb.unbound_impl(np.float64)
    ms64 = timed(lambda: one_step(impl64), steps=max(3, args.steps // 4))
    value64 = max(3, args.steps // 4) * N_WINDOWS * world / (ms64 / 1e3)
    f64_fixed = [t[6].cpu().numpy().view(np.uint64) for t in (o_dx, o_dp, o_dl, o_u)]
    del impl64
    errors = None
    if rank == 0:
        errors = output_errors(s, x, p, float(lambdas[6]), {"f32": f32_fixed, "f64": f64_fixed})

    # end to end through the C-ABI host entry (pinned host buffers, copies inside)
    hx = torch.as_tensor(x).pin_memory().numpy()
    hp = torch.as_tensor(p).pin_memory().numpy()
    hb = torch.as_tensor(s.box).pin_memory().numpy()
    hl = torch.as_tensor(lambdas).pin_memory().numpy()
    outs = [
        torch.zeros(sh, dtype=torch.int64).pin_memory().numpy().view(np.uint64)
        for sh in [(K, N, 3), (K, p.size), (K, N), (K, N)]
    ]

    def host_step():
        _lib.check(
            lib.tmnb_potential_execute_windows_host(
                impl.handle, N, p.size, hx.ctypes.data_as(ctypes.c_void_p), hp.ctypes.data_as(ctypes.c_void_p),
                hb.ctypes.data_as(ctypes.c_void_p), K, hl.ctypes.data_as(ctypes.c_void_p),
                *[o.ctypes.data_as(ctypes.c_void_p) for o in outs],
            )
        )

    for _ in range(max(1, args.warmup)):
        host_step()
    e2e_steps = max(3, args.steps // 2)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        host_step()
    t1 = time.perf_counter()
    barrier(world)
    e2e_s = max_over_ranks(t1 - t0, world)
    e2e_value = e2e_steps * N_WINDOWS * world / e2e_s
    h2d = hx.nbytes + hp.nbytes + hb.nbytes + hl.nbytes
    d2h = sum(o.nbytes for o in outs)

    # check/prepare, 5 rebuild-chain kernels (returning at once unless rebuilding), dep tiles, pair, finalize
    launches_per_step = 9
    result = {
        "metric": "nonbonded evals/s at 22,840 atoms (u, du_dx, du_dp, du_dl; 12 lambda windows per step)",
        "value": value,
        "unit": "evals/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 pair arithmetic, int64 fixed-point accumulation",
        "data": "synthetic (seeded water + ligand box; DHFR needs OpenMM)",
        "config": {
            "workload": "water_ligand_22840: 7,600 waters + 40-atom ligand, 6.1 nm box, 12 lambda windows per call",
            "atoms": N,
            "exclusions": int(n_excl),
            "pairs_in_cutoff_per_eval": int(np.mean([c[0] for c in counts])),
            "nblist_tiles": tiles,
            "nblist_items": items,
            "l2": "flushed before every timed step (256 MiB write)",
            "parallelism": f"replicas x{world}",
            "pairs_per_multi_window_launch": int(shared[0]),
            "errors_vs_fp64_oracle": errors,
        },
        "e2e": {"value": e2e_value, "unit": "evals/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": launches_per_step * args.steps,
        "roofline": {
            "bound": "fp32",
            "achieved": achieved,
            "peak": peak.value,
            "unit": "TFLOP/s",
            "frac": achieved / peak.value,
            # dram__bytes_read.sum + dram__bytes_write.sum of one launch of this kernel on
            # this workload (ncu capture, k_pair_12windows_water_ligand_22840.md under
            # profiles/): the working set stays in L2, DRAM is not the bound
            "traffic": PAIR_LAUNCH_DRAM_BYTES,
            "traffic_unit": "bytes per launch",
            "kernel": "k_pair (full variant, 12 windows in one launch)",
            "pair_kernel_ms": float(np.mean(pair_ms)),
            "flops_per_launch": float(flops_launch),
            "flops_per_pair": {"plain": FLOPS_PER_PAIR, "lj_extra": FLOPS_PER_LJ_PAIR,
                               "lambda_dependent_extra": FLOPS_PER_ALCH_PAIR},
            "peak_source": "FP32 FMA throughput measured by tmnb_probe_fp32_peak on this GPU",
            "hbm": {"peak_gbs": hbm_peak, "peak_source": "hbm_gbs of MEASURED_PEAKS.json (copy bandwidth)",
                    "stages": hbm},
        },
        "single_window_calls": {
            "value": seq_value,
            "unit": "evals/s",
            "ms_per_step": seq_ms / args.steps,
            "pair_kernel_ms": float(np.mean(pair_ms_single)),
            "achieved_tflops": achieved_single,
            "note": "the same 12 windows as 12 tmnb_potential_execute_device calls",
        },
        "fp64": {
            "value": value64,
            "unit": "evals/s",
            "ms_per_step": ms64 / max(3, args.steps // 4),
            "note": "the same 12-window call through unbound_impl(np.float64) (FP64 pair arithmetic)",
        },
    }
    try:
        result["md"] = run_md_tmnb()
        result["ns_per_day"] = result["md"]["ns_per_day"]
    except Exception as e:  # report, do not hide the evaluation numbers
        result["md"] = {"error": str(e)[:300]}
    forms = [f for f in args.forms.split(",") if f]
    if "batch" in forms:
        try:
            result["batch"] = run_batch_form()
        except Exception as e:
            result["batch"] = {"error": str(e)[:300]}
    if "serve" in forms:
        try:
            result["serve"] = run_serve_form()
        except Exception as e:
            result["serve"] = {"error": str(e)[:300]}
    if "grad" in forms:
        try:
            result["grad"] = run_grad_form()
        except Exception as e:
            result["grad"] = {"error": str(e)[:300]}
    clk.__exit__()
    result["clocks"] = clk.summary()
    return result


def summary(res):
    """The headline numbers of every form, flat, for the end of the JSON line."""
    def get(d, *ks):
        for k in ks:
            if not isinstance(d, dict) or k not in d:
                return None
            d = d[k]
        return d

    err = get(res, "config", "errors_vs_fp64_oracle") or {}
    out = {
        "evals_per_s_12_windows": res.get("value"),
        "evals_per_s_single_calls": get(res, "single_window_calls", "value"),
        "evals_per_s_fp64_12_windows": get(res, "fp64", "value"),
        "e2e_evals_per_s": get(res, "e2e", "value"),
        "md_ns_per_day": get(res, "md", "ns_per_day"),
        "pair_kernel_fp32_frac": get(res, "roofline", "frac"),
        "batch_eval_speedup_vs_512_plain": get(res, "batch", "speedup_vs_plain"),
        "batch_md_speedup_vs_512_plain": get(res, "batch", "md", "speedup_vs_plain_evals"),
        "batch_windows_grouped_speedup_vs_512_plain": get(res, "batch", "windows_grouped", "speedup_vs_plain"),
        "serve_throughput_rps": get(res, "serve", "throughput_requests_per_s"),
        "serve_eval_p50_ms": None,
        "serve_eval_p99_ms": None,
        "serve_md_p50_s": get(res, "serve", "latency_md", "p50_s"),
        "serve_md_p99_s": get(res, "serve", "latency_md", "p99_s"),
        "grad_ms": get(res, "grad", "ms_per_loss_gradient"),
    }
    p50 = get(res, "serve", "latency_eval", "p50_s")
    p99 = get(res, "serve", "latency_eval", "p99_s")
    out["serve_eval_p50_ms"] = None if p50 is None else p50 * 1e3
    out["serve_eval_p99_ms"] = None if p99 is None else p99 * 1e3
    for prec in ("f32", "f64"):
        for k, v in (err.get(prec) or {}).items():
            out[f"err_{prec}_{k}"] = v
    for name, v in (get(res, "roofline", "hbm", "stages") or {}).items():
        out[f"hbm_frac_{name.split(' ')[0]}"] = v["frac"]
    return out


MD_STEPS = 10000
MD_DT = 2.5e-3
MD_EQ_STEPS = 2000
MD_EQ_DT = 0.5e-3
MD_LAMBDA = 0.5
MD_TEMPERATURE = 300.0
MD_BARO_INTERVAL = 25


def md_system():
    from timemachine_b200 import testsystems

    return testsystems.water_ligand_23k(seed=SEED, hmr=True)


def md_groups(s):
    return [np.flatnonzero(s.group_of == g) for g in range(int(s.group_of.max()) + 1)]


def md_v0(s, seed=SEED):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(s.N, 3)) * np.sqrt(0.008314462618 * MD_TEMPERATURE / s.masses)[:, None]


def run_md_tmnb(steps=MD_STEPS):
    """configs[1] MD: 10,000 Langevin steps at 2.5 fs (HMR, H = 3 amu), MC barostat
    every 25 steps at 1 bar, lambda 0.5, from a state equilibrated at 0.5 fs."""
    from timemachine_b200 import md
    from timemachine_b200 import potentials as P

    s = md_system()
    nb = P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    bps = [
        P.HarmonicBond(s.bond_idxs).bind(s.bond_params).bound_impl(np.float32),
        P.HarmonicAngle(s.angle_idxs).bind(s.angle_params).bound_impl(np.float32),
        nb.bind(s.params).bound_impl(np.float32),
    ]
    baro = md.MonteCarloBarostat(s.N, 1.0, MD_TEMPERATURE, md_groups(s), MD_BARO_INTERVAL, SEED + 1)
    eq = md.Context(s.x, md_v0(s), s.box, md.LangevinIntegrator(MD_TEMPERATURE, MD_EQ_DT, 1.0, s.masses, SEED), bps, baro)
    eq.multiple_steps(np.full(MD_EQ_STEPS, MD_LAMBDA))
    x, v, box = eq.get_x_t(), eq.get_v_t(), eq.get_box()
    del eq
    ctx = md.Context(x, v, box, md.LangevinIntegrator(MD_TEMPERATURE, MD_DT, 1.0, s.masses, SEED + 7), bps, baro)
    ctx.multiple_steps(np.full(200, MD_LAMBDA))  # warm-up (graph capture)
    lam = np.full(steps, MD_LAMBDA)
    t0 = time.perf_counter()
    ctx.multiple_steps(lam)
    dt_wall = time.perf_counter() - t0
    xf = ctx.get_x_t()
    acc, att, _ = ctx.barostat_stats()
    steps_per_s = steps / dt_wall
    return {
        "ns_per_day": steps_per_s * MD_DT * 86400 / 1000,
        "steps_per_s": steps_per_s,
        "steps": steps,
        "dt_ps": MD_DT,
        "lambda": MD_LAMBDA,
        "barostat": {"interval": MD_BARO_INTERVAL, "attempted": att, "accepted": acc},
        "finite": bool(np.all(np.isfinite(xf))),
        "timing": "wall clock around Context.multiple_steps (ends with a stream synchronise)",
        "potentials": "HarmonicBond + HarmonicAngle + Nonbonded (22,840 atoms)",
    }


def run_md_reference(steps=MD_STEPS):
    """The same MD through the reference runtime (Context/LangevinIntegrator/MonteCarloBarostat)."""
    from oracle.refgpu import refgpu
    from timemachine_b200.md import langevin_coefficients

    s = md_system()
    ref = refgpu.RefNonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    group_of = s.group_of

    def make(x, v, box, dt, seed):
        ca, cb, cc = langevin_coefficients(MD_TEMPERATURE, dt, 1.0, s.masses)
        return refgpu.RefMD(
            ref, s.params, x, v, box, dt, ca, -cb, cc, seed, 1.0, MD_TEMPERATURE, group_of, MD_BARO_INTERVAL,
            s.bond_idxs, s.bond_params, s.angle_idxs, s.angle_params,
        )

    eq = make(s.x, md_v0(s), s.box, MD_EQ_DT, SEED)
    x, box = eq.run(MD_EQ_STEPS, MD_LAMBDA)
    del eq
    m = make(x, md_v0(s, SEED + 3), box, MD_DT, SEED + 7)
    m.run(200, MD_LAMBDA)
    t0 = time.perf_counter()
    xf, _ = m.run(steps, MD_LAMBDA)
    dt_wall = time.perf_counter() - t0
    steps_per_s = steps / dt_wall
    return {
        "ns_per_day": steps_per_s * MD_DT * 86400 / 1000,
        "steps_per_s": steps_per_s,
        "steps": steps,
        "finite": bool(np.all(np.isfinite(xf))),
        "timing": "wall clock around Context.multiple_steps",
    }


BATCH_SYSTEMS = 64
BATCH_WINDOWS = 8
BATCH_CHUNK = 500
BATCH_MD = dict(temperature=300.0, dt=1.5e-3, friction=1.0)


def batch_workload(seed=SEED):
    """64 water + ligand systems, sizes log-uniform on [1,500, 30,000] atoms at
    1 g/cm^3, ligands of 20-60 atoms; 8 lambda windows each (512 replicas)."""
    from timemachine_b200 import testsystems

    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(1500), np.log(30000), BATCH_SYSTEMS)).astype(int)
    systems = [testsystems.system_of_size(int(n), seed=seed + 17 * k) for k, n in enumerate(sizes)]
    return systems, np.linspace(0.0, 1.0, BATCH_WINDOWS)


def _mb_velocities(rng, s, temperature):
    return rng.normal(size=(s.N, 3)) * np.sqrt(0.008314462618 * temperature / s.masses)[:, None]


def run_batch_form():
    """Batching form: 512 replicas (64 systems x 8 windows) through one launch
    sequence per step, against 512 sequential plain calls (one Nonbonded +
    HarmonicBond + HarmonicAngle execute_device per replica), and one
    CUDA-graph-captured 500-step MD chunk of all replicas."""
    import torch

    from timemachine_b200 import potentials as P
    from timemachine_b200.batch import ReplicaBatch

    systems, lambdas = batch_workload()
    n_rep = len(systems) * len(lambdas)
    atoms = int(sum(s.N for s in systems) * len(lambdas))
    b = ReplicaBatch()
    rng = np.random.default_rng(SEED + 5)
    for k, s in enumerate(systems):
        for w, lam in enumerate(lambdas):
            b.add(s, lam, v=_mb_velocities(rng, s, BATCH_MD["temperature"]), md=BATCH_MD, seed=1000 * k + w)
    stream = torch.cuda.ExternalStream(b.stream)

    def timed(fn, reps):
        fn()  # warm-up (rebuilds, graph capture)
        b.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3

    tune_best, tune_table = b.autotune(
        mode="eval",
        steps=2,
        repeats=1,
        candidates=[
            dict(chunk=c, padding=p, grid_bits_offset=0, pair_ctas_per_sm=0, rows=r)
            for r in (8, 16, 32) for c in (8, 16, 32, 64, 128) for p in (0.06, 0.1)
        ],
    )
    t_eval = timed(lambda: b.evaluate(), 3)
    batch_evals = 3 * n_rep / t_eval

    # 512 sequential plain calls, device-resident inputs, CUDA events on the torch stream
    cur = torch.cuda.current_stream()
    plain = []
    for s in systems:
        pots = [
            (P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
             .unbound_impl(np.float32), s.params),
            (P.HarmonicBond(s.bond_idxs).unbound_impl(np.float32), s.bond_params),
            (P.HarmonicAngle(s.angle_idxs).unbound_impl(np.float32), s.angle_params),
        ]
        dev = [(impl, torch.as_tensor(np.ascontiguousarray(p), device="cuda").reshape(-1)) for impl, p in pots]
        dx = torch.as_tensor(s.x, device="cuda")
        db = torch.as_tensor(s.box, device="cuda")
        outs = [torch.zeros(sh, dtype=torch.int64, device="cuda") for sh in [(s.N, 3), (s.N * 3,), (s.N,), (s.N,)]]
        plain.append((dev, dx, db, outs))

    def plain_pass():
        for dev, dx, db, outs in plain:
            for lam in lambdas:
                for o in outs:
                    o.zero_()
                nb_impl, nb_p = dev[0]
                nb_impl.execute_device(dx, nb_p, db, float(lam), *outs, stream=cur)
                for impl, p in dev[1:]:
                    impl.execute_device(dx, p, db, float(lam), outs[0], None, None, outs[3], stream=cur)

    plain_pass()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(cur)
    plain_pass()
    e1.record(cur)
    e1.synchronize()
    t_plain = e0.elapsed_time(e1) / 1e3
    plain_evals = n_rep / t_plain

    # the same 512 evaluations with the 8 windows of each system in one
    # multi-window call (64 calls): the replicas of a system share their
    # coordinates here, so its lambda-independent tiles are evaluated once
    win_outs = {}
    for k, (dev, dx, db, outs) in enumerate(plain):
        N = dx.shape[0]
        win_outs[k] = [torch.zeros((len(lambdas),) + tuple(o.shape), dtype=torch.int64, device="cuda") for o in outs]

    def windows_pass():
        for k, (dev, dx, db, outs) in enumerate(plain):
            w = win_outs[k]
            for o in w:
                o.zero_()
            nb_impl, nb_p = dev[0]
            nb_impl.execute_windows_device(dx, nb_p, db, lambdas, *w, stream=cur)
            for impl, p in dev[1:]:
                for li, lam in enumerate(lambdas):
                    impl.execute_device(dx, p, db, float(lam), w[0][li], None, None, w[3][li], stream=cur)

    windows_pass()
    torch.cuda.synchronize()
    e0.record(cur)
    windows_pass()
    e1.record(cur)
    e1.synchronize()
    t_windows = e0.elapsed_time(e1) / 1e3
    windows_evals = n_rep / t_windows
    del plain, win_outs

    # the MD step computes forces only: its best schedule can differ from the evaluation's
    md_tune_best, md_tune_table = b.autotune(
        mode="md",
        steps=20,
        repeats=1,
        candidates=[
            dict(chunk=c, padding=p, grid_bits_offset=0, pair_ctas_per_sm=0, rows=r)
            for r in (8, 16, 32) for c in (8, 16, 32, 64, 128) for p in (0.06, 0.1)
        ],
    )
    t_md = timed(lambda: b.md(BATCH_CHUNK, chunk=BATCH_CHUNK, use_graph=True), 1)
    md_replica_steps = n_rep * BATCH_CHUNK / t_md
    sample = b.ids()[:: max(1, n_rep // 16)]
    finite = all(np.all(np.isfinite(b.get_x(r))) for r in sample)
    return {
        "workload": f"{len(systems)} water+ligand systems of {min(s.N for s in systems)}-{max(s.N for s in systems)} "
        f"atoms (log-uniform on [1500, 30000]) x {len(lambdas)} lambda windows = {n_rep} replicas, "
        f"{atoms} replica-atoms; nonbonded + harmonic bonds/angles",
        "evals_per_s": batch_evals,
        "plain_sequential_evals_per_s": plain_evals,
        "speedup_vs_plain": batch_evals / plain_evals,
        "windows_grouped": {
            "evals_per_s": windows_evals,
            "speedup_vs_plain": windows_evals / plain_evals,
            "note": "the 8 windows of each system in one multi-window call (64 calls; replicas share coordinates "
            "at this evaluation, so lambda-independent tiles are evaluated once per system)",
        },
        "eval_ms": t_eval / 3 * 1e3,
        "plain_ms": t_plain * 1e3,
        "md": {
            "replica_steps_per_s": md_replica_steps,
            "speedup_vs_plain_evals": md_replica_steps / plain_evals,
            "chunk_steps": BATCH_CHUNK,
            "chunk_ms": t_md * 1e3,
            "dt_ps": BATCH_MD["dt"],
            "aggregate_ns_per_day": md_replica_steps * BATCH_MD["dt"] * 86400 / 1000,
            "finite": bool(finite),
            "timing": "CUDA events on the batch stream around one graph-replayed 500-step chunk",
        },
        "autotune": {"best": tune_best, "candidates": [[c, t] for c, t in tune_table]},
        "autotune_md": {"best": md_tune_best, "candidates": [[c, t] for c, t in md_tune_table]},
        "timing": "CUDA events (batch stream / torch stream), inputs resident on the device",
        "device_bytes": b.bytes_in_use(),
    }


SERVE_RATE = 200.0  # requests/s
SERVE_SECONDS = 60.0  # arrival window of the serving stream
SERVE_COMPARE_SECONDS = 3.0  # prefix of the stream served both ways for the sequential comparison
SERVE_MD_STEPS = 1000
SERVE_SIZE_LEVELS = 64  # distinct system sizes (log-spaced on [500, 50000]) the stream draws from


def serve_workload(seed=SEED + 11, seconds=SERVE_SECONDS):
    """Poisson arrivals at 200/s; 70 % single evaluations, 30 % 1,000-step
    Langevin segments; sizes log-uniform on [500, 50,000] atoms (drawn from 64
    log-spaced levels, so that the stream's systems are built once each);
    lambda U(0, 1)."""
    from timemachine_b200 import testsystems
    from timemachine_b200.serve import Request

    rng = np.random.default_rng(seed)
    levels = np.exp(np.linspace(np.log(500), np.log(50000), SERVE_SIZE_LEVELS)).astype(int)
    built = {}
    t, reqs = 0.0, []
    while True:
        t += rng.exponential(1.0 / SERVE_RATE)
        if t > seconds:
            break
        n = int(np.exp(rng.uniform(np.log(500), np.log(50000))))
        n = int(levels[np.argmin(np.abs(np.log(levels) - np.log(n)))])
        if n not in built:
            built[n] = testsystems.system_of_size(n, seed=int(rng.integers(1 << 30)))
        s = built[n]
        kind = "md" if rng.uniform() < 0.3 else "eval"
        reqs.append(
            Request(
                rid=len(reqs), system=s, lam=float(rng.uniform()), kind=kind, arrival=t,
                n_steps=SERVE_MD_STEPS if kind == "md" else 0,
                v0=_mb_velocities(rng, s, BATCH_MD["temperature"]) if kind == "md" else None,
                seed=int(rng.integers(1 << 30)), md=BATCH_MD,
            )
        )
    return reqs


def run_serve_form():
    """Serving form: the 60 s request stream of the serving workload through
    the continuous-batching server; and its first 3 s both through the server
    and through sequential plain calls on the same GPU (the comparison)."""
    import dataclasses

    from timemachine_b200.serve import Server, latency_stats, run_sequential

    reqs = serve_workload()
    md_atom_steps = sum(r.system.N * r.n_steps for r in reqs if r.kind == "md")
    server = Server(hbm_budget_bytes=150e9, md_chunk=50)
    t0 = time.perf_counter()
    done = server.run(reqs)
    wall = time.perf_counter() - t0
    evals = [r for r in done if r.kind == "eval"]
    mds = [r for r in done if r.kind == "md"]
    # the comparison: the first seconds of the same stream, served both ways
    prefix = [r for r in serve_workload(seconds=SERVE_COMPARE_SECONDS)]
    fresh = [dataclasses.replace(r) for r in prefix]
    s2 = Server(hbm_budget_bytes=150e9, md_chunk=50)
    t1 = time.perf_counter()
    done2 = s2.run(prefix)
    wall2 = time.perf_counter() - t1
    seq = run_sequential(fresh)
    seq_wall = max(r.finished for r in seq) - min(r.arrival for r in seq)
    return {
        "workload": f"{len(reqs)} requests over {SERVE_SECONDS:.0f} s of Poisson arrivals at {SERVE_RATE:.0f}/s "
        f"({len(evals)} evaluations, {len(mds)} x {SERVE_MD_STEPS}-step MD segments), sizes log-uniform on "
        "[500, 50000] atoms (64 levels), lambda U(0,1), 150 GB HBM budget",
        "latency": latency_stats(done),
        "latency_eval": latency_stats(evals) if evals else None,
        "latency_md": latency_stats(mds) if mds else None,
        "throughput_requests_per_s": len(done) / wall,
        "wall_s": wall,
        "offered_requests_per_s": len(reqs) / SERVE_SECONDS,
        "offered_md_atom_steps_per_s": md_atom_steps / SERVE_SECONDS,
        "served_md_atom_steps_per_s": md_atom_steps / wall,
        "capacity_note": "the stream offers more MD work than one B200 serves in 60 s when served_md_atom_steps_per_s "
        "< offered_md_atom_steps_per_s; the backlog then sets the MD latencies, not the loop",
        "eval_launches": server.ev.launched,
        "md_launches": server.md.launched,
        "peak_device_bytes": server.peak_bytes,
        "compare_prefix": {
            "requests": len(prefix),
            "seconds_of_arrivals": SERVE_COMPARE_SECONDS,
            "server": {"latency_eval": latency_stats([r for r in done2 if r.kind == "eval"]),
                       "latency_md": latency_stats([r for r in done2 if r.kind == "md"]),
                       "throughput_requests_per_s": len(done2) / wall2, "wall_s": wall2},
            "sequential_plain": {"latency_eval": latency_stats([r for r in seq if r.kind == "eval"]),
                                 "latency_md": latency_stats([r for r in seq if r.kind == "md"]),
                                 "throughput_requests_per_s": len(seq) / seq_wall, "wall_s": seq_wall},
        },
        "timing": "host wall clock from each request's arrival to its result on the host (D2H included)",
    }


GRAD_FRAMES = 32
GRAD_LAMBDA = 0.5


def grad_workload(n_frames=GRAD_FRAMES):
    """The differentiation workload: (loss_and_grads, parts). loss_and_grads()
    runs the forward kernels and the adjoint kernel over all frames and returns
    (loss, d/dparams, d/doffsets); parts holds the system, the potential, the
    frames (host and device), the ligand atoms, the box, the target forces and
    the base w offsets."""
    import torch

    from timemachine_b200 import potentials as P
    from timemachine_b200 import testsystems
    from timemachine_b200.adjoint import nonbonded_forces

    s = testsystems.build_system(1650, (1650 * testsystems.WATER_VOLUME) ** (1 / 3), seed=SEED + 3, n_ligand=50)
    lig = np.flatnonzero(s.lambda_offset_idxs != 0)
    rng = np.random.default_rng(SEED + 4)
    frames = [s.x + rng.normal(scale=0.01, size=s.x.shape) for _ in range(n_frames)]
    impl = P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    impl = impl.unbound_impl(np.float32)
    p_target = s.params.copy()
    p_target[lig] *= 1 + 0.05 * rng.normal(size=(lig.size, 3))
    box = torch.as_tensor(s.box, device="cuda")
    xs = [torch.as_tensor(f, device="cuda") for f in frames]
    targets = []
    with torch.no_grad():
        pt = torch.as_tensor(p_target, device="cuda")
        w0 = torch.as_tensor(s.lambda_offset_idxs.astype(np.float64), device="cuda")
        for x in xs:
            targets.append(nonbonded_forces(impl, pt, w0, x, box, GRAD_LAMBDA)[0].clone())

    def loss_and_grads():
        params = torch.as_tensor(s.params, device="cuda").requires_grad_(True)
        w_off = torch.as_tensor(s.lambda_offset_idxs.astype(np.float64), device="cuda").requires_grad_(True)
        total = 0.0
        for x, t in zip(xs, targets):
            f, dl = nonbonded_forces(impl, params, w_off, x, box, GRAD_LAMBDA)
            total = total + ((f - t) ** 2).mean() + 0.1 * dl**2
        loss = total / len(xs)
        loss.backward()
        return loss, params.grad, w_off.grad

    return loss_and_grads, dict(s=s, impl=impl, frames=frames, lig=lig, xs=xs, box=box, targets=targets, w0=w0)


def run_grad_form():
    """Differentiation form: 1,650 waters + a 50-atom ligand; 32 frames
    (Gaussian perturbations of 0.01 nm); targets = forces with the ligand
    parameters perturbed by 5 %; loss = mean squared force error + 0.1 du_dl^2
    at lambda 0.5; gradients with respect to the ligand's charges, sigmas,
    sqrt(eps) and w offsets through the adjoint kernel. Checked against the
    FP64 double-backward oracle and FP64 central differences (step 1e-4) on
    one frame."""
    import torch

    from oracle.nonbonded_oracle import Oracle, candidate_pairs, force_vjp_oracle
    from timemachine_b200.adjoint import nonbonded_forces

    loss_and_grads, parts = grad_workload()
    s, impl, frames, lig = parts["s"], parts["impl"], parts["frames"], parts["lig"]
    xs, box, targets, w0 = parts["xs"], parts["box"], parts["targets"], parts["w0"]
    loss_and_grads()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    loss, gp, gw = loss_and_grads()
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1)

    # FP64 references on frame 0 (one frame of the loss, same upstream form)
    x0 = frames[0]
    f0, dl0 = nonbonded_forces(impl, torch.as_tensor(s.params, device="cuda"), w0, xs[0], box, GRAD_LAMBDA)
    o = Oracle(s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff, s.exclusion_idxs, s.scales)
    fx, _, fl, _ = o(x0, s.params, s.box, GRAD_LAMBDA)
    t0 = targets[0].cpu().numpy()
    G = 2.0 * (fx - t0) / fx.size
    g = 0.2 * fl
    pairs = candidate_pairs(x0, s.box, s.cutoff)
    off = s.lambda_offset_idxs.astype(np.float64)
    _, rp, rw = force_vjp_oracle(
        x0, s.params, s.box, GRAD_LAMBDA, s.lambda_plane_idxs, off, s.beta, s.cutoff, s.exclusion_idxs, s.scales, G, g,
        pairs=pairs,
    )
    # the kernel's VJP with the same (FP64) upstream gradients
    kp = torch.zeros(s.params.size, dtype=torch.float64, device="cuda")
    kw = torch.zeros(s.N, dtype=torch.float64, device="cuda")
    impl.adjoint_device(xs[0], torch.as_tensor(s.params, device="cuda").reshape(-1), box, GRAD_LAMBDA,
                        torch.as_tensor(G, device="cuda"), g, kp, kw)
    kp = kp.cpu().numpy().reshape(-1, 3)
    kw = kw.cpu().numpy()

    def rel(a, b):
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

    h = 1e-4

    def phi(params, offsets):
        return force_vjp_oracle(x0, params, s.box, GRAD_LAMBDA, s.lambda_plane_idxs, offsets, s.beta, s.cutoff,
                                s.exclusion_idxs, s.scales, G, g, pairs=pairs)[0]

    def crosses_cutoff(a):
        # a +-h offset step that carries a pair across the (discontinuous) cutoff is not a derivative test
        mine = pairs[(pairs[:, 0] == a) | (pairs[:, 1] == a)]
        i, j = mine[:, 0], mine[:, 1]
        L = np.diag(s.box)
        r = x0[i] - x0[j]
        r -= L * np.floor(r / L + 0.5)
        inside = []
        for dh in (-h, h):
            o = off.copy()
            o[a] += dh
            w = s.cutoff * (s.lambda_plane_idxs + o * GRAD_LAMBDA)
            inside.append(np.sqrt((r * r).sum(1) + (w[i] - w[j]) ** 2) < s.cutoff)
        return np.any(inside[0] != inside[1])

    fd_err, n_fd = 0.0, 0
    for a in lig[:3]:
        for col in range(3):
            pp, pm = s.params.copy(), s.params.copy()
            pp[a, col] += h
            pm[a, col] -= h
            fd = (phi(pp, off) - phi(pm, off)) / (2 * h)
            fd_err = max(fd_err, abs(fd - kp[a, col]) / max(abs(fd), 1.0))
            n_fd += 1
    for a in [a for a in lig if not crosses_cutoff(a)][:3]:
        op, om = off.copy(), off.copy()
        op[a] += h
        om[a] -= h
        fd = (phi(s.params, op) - phi(s.params, om)) / (2 * h)
        fd_err = max(fd_err, abs(fd - kw[a]) / max(abs(fd), 1.0))
        n_fd += 1
    return {
        "workload": f"{s.N} atoms (1650 waters + 50-atom ligand), {GRAD_FRAMES} frames, lambda {GRAD_LAMBDA}; "
        "loss = mean squared force error + 0.1 du_dl^2; d/d ligand (q, sigma, sqrt eps, w offset)",
        "loss": float(loss.detach()),
        "ms_per_loss_gradient": ms,
        "frames_per_s": GRAD_FRAMES / (ms / 1e3),
        "grad_norm_ligand_params": float(gp[lig].norm()),
        "grad_norm_ligand_offsets": float(gw[lig].norm()),
        "vjp_relative_error_vs_fp64_double_backward": {"params": rel(kp, rp), "offsets": rel(kw, rw)},
        "vjp_max_relative_error_vs_fp64_central_differences_step_1e-4": fd_err,
        "central_difference_checks": n_fd,
        "timing": "CUDA events around the 32-frame loss and its backward (forward kernels + adjoint kernel)",
    }


def cpu_baseline(x, p, s, lambdas, n_evals=2):
    import torch

    from oracle.nonbonded_oracle import Oracle

    cores = len(os.sched_getaffinity(0))
    torch.set_num_threads(cores)
    o = Oracle(s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff, s.exclusion_idxs, s.scales)
    pairs = o.pairs(x, s.box)
    o(x, p, s.box, float(lambdas[0]), pairs)  # warm-up
    t0 = time.perf_counter()
    for k in range(n_evals):
        o(x, p, s.box, float(lambdas[k % len(lambdas)]), pairs)
    dt = time.perf_counter() - t0
    return n_evals / dt, cores


def run_reference(args, world, rank, local):
    if rank != 0:
        return None
    s, x, p, lambdas = build_workload(0)
    import torch

    from oracle.nonbonded_oracle import Oracle

    cores = len(os.sched_getaffinity(0))
    torch.set_num_threads(cores)
    o = Oracle(s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff, s.exclusion_idxs, s.scales)
    pairs = o.pairs(x, s.box)
    for k in range(args.warmup):
        o(x, p, s.box, float(lambdas[k % N_WINDOWS]), pairs)
    t0 = time.perf_counter()
    for k in range(args.steps):
        o(x, p, s.box, float(lambdas[k % N_WINDOWS]), pairs)
    dt = time.perf_counter() - t0
    value = args.steps / dt
    result = {
        "impl": "reference",
        "metric": "nonbonded evals/s at 22,840 atoms (u, du_dx, du_dp, du_dl; 12 lambda windows per step)",
        "value": value,
        "unit": "evals/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded water + ligand box)",
        "config": {"workload": "water_ligand_22840, one lambda window per step", "atoms": s.N},
        "cpu_baseline": {
            "value": value,
            "unit": "evals/s",
            "cores": cores,
            "kind": "port",
            "sample": f"{args.steps} single-window evaluations of the 22,840-atom box (FP64 torch restatement of nonbonded_v3; jax absent)",
        },
        "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    try:
        result["reference_gpu"] = reference_gpu(s, x, p, lambdas, args)
    except Exception as e:
        result["reference_gpu"] = {"unavailable": str(e)[:200]}
    return result


def reference_gpu(s, x, p, lambdas, args):
    """The reference CUDA build (oracle/_ref) on the same workload, device-resident."""
    import torch

    from oracle.refgpu import refgpu

    if not refgpu.available() or not torch.cuda.is_available():
        return {"unavailable": "reference CUDA build (oracle/_ref) not present"}
    ref = refgpu.RefNonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
    N = s.N
    dx = torch.as_tensor(x, device="cuda")
    dp = torch.as_tensor(p, device="cuda").reshape(-1)
    db = torch.as_tensor(s.box, device="cuda")
    outs = [torch.zeros(sh, dtype=torch.int64, device="cuda") for sh in [(N, 3), (p.size,), (N,), (N,)]]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    def step():
        for lam in lambdas:
            for o in outs:
                o.zero_()
            ref.execute_device(dx, dp, db, float(lam), *outs, stream=stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.zero_()
        evs[k][0].record()
        step()
        evs[k][1].record()
    torch.cuda.synchronize()
    total_ms = sum(a.elapsed_time(b) for a, b in evs)
    # host entry (the reference's execute_host allocates and copies every call)
    t0 = time.perf_counter()
    n_host = max(3, args.steps // 2)
    for _ in range(n_host):
        for lam in lambdas:
            ref.execute_host_fixed(x, p, s.box, float(lam))
    t1 = time.perf_counter()
    try:
        md_ref = run_md_reference()
    except Exception as e:
        md_ref = {"error": str(e)[:300]}
    return {
        "value": args.steps * N_WINDOWS / (total_ms / 1e3),
        "unit": "evals/s",
        "ms_per_step": total_ms / args.steps,
        "e2e_value": n_host * N_WINDOWS / (t1 - t0),
        "md": md_ref,
        "source": "reference timemachine CUDA sources built for sm_100a (FanoutSummedPotential[NonbondedAllPairs_f32, NonbondedPairList_f32_negated])",
    }


def main():
    args = parse()
    world, rank, local = dist_setup()
    if args.profile:
        run_profile(args, local)
        return
    if args.impl == "reference":
        res = run_reference(args, world, rank, local)
    else:
        res = run_tmnb(args, world, rank, local)
        if rank == 0:
            s, x, p, lambdas = build_workload(0)
            v, cores = cpu_baseline(x, p, s, lambdas)
            res["cpu_baseline"] = {
                "value": v,
                "unit": "evals/s",
                "cores": cores,
                "kind": "port",
                "sample": "2 single-window evaluations of the 22,840-atom box by the FP64 oracle (all host threads)",
            }
    if rank == 0 and res is not None:
        if args.impl != "reference":
            res["summary"] = summary(res)  # last key: the headline numbers of every form
        print(json.dumps(res))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
