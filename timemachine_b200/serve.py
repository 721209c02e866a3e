"""Serving loop: continuous batching of energy/force and short-MD requests.

Requests of different atom counts arrive over time. The loop keeps each
admitted request's coordinates, velocities, box and neighbour list resident
on the device (one replica of a ReplicaBatch), admits waiting requests as
device memory frees up (admission by HBM footprint against a budget), and
serves every admitted request together: each loop iteration launches one
batched evaluation of the waiting energy/force requests and one batched chunk
of MD steps of the running segments, on two streams, so their work overlaps
on the device. Requests that arrive while others are on the GPU join at the
next iteration.

A request's result does not depend on what else is being served: each replica
is an independent system with integer (fixed-point) accumulation, so it is
bit-identical alone and in any mix.
"""

import time
from dataclasses import dataclass, field

import numpy as np

from .batch import ReplicaBatch


@dataclass
class Request:
    """kind "eval": one (du_dx, du_dp, du_dl, u) evaluation; kind "md": n_steps
    Langevin steps from (system.x, v0), returning the final (x, v)."""

    rid: int
    system: object
    lam: float
    kind: str
    arrival: float = 0.0
    n_steps: int = 0
    v0: np.ndarray = None
    seed: int = 0
    md: dict = None
    # filled by the server
    admitted: float = None
    finished: float = None
    result: tuple = None
    steps_done: int = 0
    _replica: int = field(default=None, repr=False)


def _terms(system, name):
    a = getattr(system, name, None)
    return 0 if a is None else len(a)


class Server:
    def __init__(self, hbm_budget_bytes=150e9, md_chunk=50, tuning=None):
        self.budget = float(hbm_budget_bytes)
        self.md_chunk = int(md_chunk)
        self.eval_engine = ReplicaBatch()
        self.md_engine = ReplicaBatch()
        if tuning:
            self.eval_engine.set_tuning(**tuning)
            self.md_engine.set_tuning(**tuning)
        self.waiting = []
        self.active_eval = []
        self.active_md = []
        self.done = []
        self.iterations = 0
        self.peak_bytes = 0

    def footprint(self, req):
        s = req.system
        return self.eval_engine.footprint(
            s.N, len(s.exclusion_idxs), _terms(s, "bond_idxs"), _terms(s, "angle_idxs")
        )

    def bytes_in_use(self):
        return self.eval_engine.bytes_in_use() + self.md_engine.bytes_in_use()

    def submit(self, req):
        self.waiting.append(req)

    def _admit(self, now):
        """FIFO admission of arrived requests while the HBM budget allows."""
        used = self.bytes_in_use()
        keep = []
        blocked = False
        for req in self.waiting:
            if blocked or req.arrival > now:
                keep.append(req)
                continue
            need = self.footprint(req)
            if used + need > self.budget:
                if need > self.budget:
                    raise RuntimeError(f"request {req.rid} needs {need} bytes, above the HBM budget")
                blocked = True  # keep arrival order
                keep.append(req)
                continue
            if req.kind == "eval":
                req._replica = self.eval_engine.add(req.system, req.lam)
                self.active_eval.append(req)
            else:
                req._replica = self.md_engine.add(req.system, req.lam, v=req.v0, md=req.md, seed=req.seed)
                self.active_md.append(req)
            req.admitted = time.perf_counter()
            used += need
        self.waiting = keep
        self.peak_bytes = max(self.peak_bytes, used)

    def step(self):
        """One loop iteration: admit, launch both engines, collect completions."""
        self._admit(time.perf_counter())
        evals = list(self.active_eval)
        if evals:
            self.eval_engine.evaluate()
        n_md = 0
        if self.active_md:
            n_md = min(self.md_chunk, min(r.n_steps - r.steps_done for r in self.active_md))
            self.md_engine.md(n_md, chunk=n_md, use_graph=False)
        if evals:
            self.eval_engine.synchronize()
            for req in evals:
                req.result = self.eval_engine.result_fixed(req._replica)
                req.finished = time.perf_counter()
                self.eval_engine.remove(req._replica)
                self.done.append(req)
            self.active_eval = []
        if n_md:
            self.md_engine.synchronize()
            still = []
            for req in self.active_md:
                req.steps_done += n_md
                if req.steps_done >= req.n_steps:
                    req.result = (self.md_engine.get_x(req._replica), self.md_engine.get_v(req._replica))
                    req.finished = time.perf_counter()
                    self.md_engine.remove(req._replica)
                    self.done.append(req)
                else:
                    still.append(req)
            self.active_md = still
        self.iterations += 1

    def busy(self):
        return bool(self.waiting or self.active_eval or self.active_md)

    def run(self, requests, t0=None):
        """Serves `requests` (arrival times in seconds relative to t0, default
        now) until all are done; returns them in completion order. A request's
        latency is finished - arrival (both absolute after this call)."""
        t0 = time.perf_counter() if t0 is None else t0
        for r in requests:
            r.arrival = t0 + r.arrival
            self.submit(r)
        while self.busy():
            if not (self.active_eval or self.active_md):
                now = time.perf_counter()
                nxt = min(r.arrival for r in self.waiting)
                if nxt > now:
                    time.sleep(min(nxt - now, 0.01))
                    continue
            self.step()
        return self.done


def run_sequential(requests, t0=None):
    """The same request stream through sequential plain calls, one request at a
    time in arrival order: an evaluation is one Nonbonded + bonded
    execute_selective, an MD segment one single-system Context. Returns the
    requests with finished times (same latency convention as Server.run)."""
    from . import md as mdmod
    from . import potentials as P

    t0 = time.perf_counter() if t0 is None else t0
    for r in requests:
        r.arrival = t0 + r.arrival
    for req in sorted(requests, key=lambda r: r.arrival):
        now = time.perf_counter()
        if req.arrival > now:
            time.sleep(req.arrival - now)
        s = req.system
        nb = P.Nonbonded(s.exclusion_idxs, s.scales, s.lambda_plane_idxs, s.lambda_offset_idxs, s.beta, s.cutoff)
        if req.kind == "eval":
            dx, dp, dl, u = nb.unbound_impl(np.float32)._execute_fixed(s.x, s.params, s.box, req.lam, True, True, True, True)
            for pot, params in [(P.HarmonicBond(s.bond_idxs), s.bond_params), (P.HarmonicAngle(s.angle_idxs), s.angle_params)]:
                bdx, _, _, bu = pot.unbound_impl(np.float32)._execute_fixed(s.x, params, s.box, req.lam, True, False, False, True)
                dx = dx + bdx
                u = u + bu
            req.result = (dx, dp.reshape(-1, 3), dl, u)
        else:
            intg = mdmod.LangevinIntegrator(
                req.md["temperature"], req.md["dt"], req.md["friction"], s.masses, req.seed
            )
            bps = [
                P.HarmonicBond(s.bond_idxs).bind(s.bond_params).bound_impl(np.float32),
                P.HarmonicAngle(s.angle_idxs).bind(s.angle_params).bound_impl(np.float32),
                nb.bind(s.params).bound_impl(np.float32),
            ]
            ctx = mdmod.Context(s.x, req.v0 if req.v0 is not None else np.zeros_like(s.x), s.box, intg, bps)
            ctx.multiple_steps(np.full(req.n_steps, req.lam))
            req.result = (ctx.get_x_t(), ctx.get_v_t())
        req.finished = time.perf_counter()
    return requests


def latency_stats(done):
    lat = np.array([r.finished - r.arrival for r in done])
    return {
        "p50_s": float(np.percentile(lat, 50)),
        "p99_s": float(np.percentile(lat, 99)),
        "mean_s": float(lat.mean()),
        "max_s": float(lat.max()),
        "count": int(lat.size),
    }
