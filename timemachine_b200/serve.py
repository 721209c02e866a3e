"""Serving loop: continuous batching of energy/force and short-MD requests.

Requests of different atom counts arrive over time. Each admitted request's
coordinates, velocities, box and neighbour list stay resident on the device
(one replica of a ReplicaBatch); admission is by HBM footprint against a
budget. Two engines serve the two request kinds on their own CUDA streams:

- the evaluation engine runs one batched evaluation of every evaluation
  request admitted since its last batch;
- the MD engine advances every running segment by chunks of Langevin steps
  (one CUDA-graph-replayed chunk while its membership is unchanged).

The loop never waits on the device. It polls a CUDA event per engine: when an
engine's launch has completed it collects that engine's finished requests,
admits the requests that arrived meanwhile (membership changes only while the
engine is idle) and launches the engine again, so evaluations are answered as
soon as their batch ends -- they do not wait for an MD chunk -- and the two
engines' work overlaps on the device. Replica arenas are allocated and freed
in stream order, so a finished request's release does not wait for the
other engine.

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


class _Engine:
    """One ReplicaBatch with its stream, its in-flight launch and its requests."""

    def __init__(self, tuning, priority=None):
        import torch

        self.batch = ReplicaBatch(priority=priority)
        if tuning:
            self.batch.set_tuning(**tuning)
        self.stream = torch.cuda.ExternalStream(self.batch.stream)
        self.event = None  # completion event of the launch in flight
        self.running = []  # requests in the launch in flight (or resident between launches)
        self.launched = 0

    def idle(self):
        return self.event is None or self.event.query()

    def mark(self):
        import torch

        self.event = torch.cuda.Event()
        self.event.record(self.stream)
        self.launched += 1


class Server:
    """hbm_budget_bytes: device bytes all resident requests may hold.
    md_budget_fraction: the share of it MD segments may hold, so that
    evaluation requests always find room (they are short-lived).
    md_max_atoms: resident MD atoms at most (FIFO admission beyond): an MD
    chunk then takes bounded time, and under a backlog the earlier segments
    finish first instead of all advancing together.
    md_pair_ctas_per_sm: CTAs per SM of the MD engine's persistent pair
    kernel (0: as many as fit). Its CTAs hold their SM slots for the whole
    kernel, so a cap below the fit leaves slots on every SM for the
    evaluation engine's kernels."""

    def __init__(self, hbm_budget_bytes=150e9, md_chunk=50, tuning=None, md_graphs=True,
                 md_budget_fraction=0.8, md_max_atoms=4_000_000, md_pair_ctas_per_sm=0):
        self.budget = float(hbm_budget_bytes)
        self.md_budget = self.budget * float(md_budget_fraction)
        self.md_max_atoms = int(md_max_atoms)
        self.md_chunk = int(md_chunk)
        self.md_graphs = md_graphs
        # evaluations are short and latency-bound: their stream gets the
        # highest scheduling priority, so their blocks go first whenever the
        # MD chunk's kernels free an SM
        self.ev = _Engine(tuning, priority=-1000)
        md_tuning = dict(tuning or {})
        if md_pair_ctas_per_sm:
            md_tuning["pair_ctas_per_sm"] = int(md_pair_ctas_per_sm)
        self.md = _Engine(md_tuning)
        self.waiting = []  # arrived or future requests, not yet admitted
        self.done = []
        self.iterations = 0
        self.peak_bytes = 0
        self.md_chunk_steps = []  # steps of each MD launch

    # kept for callers of the earlier interface
    @property
    def eval_engine(self):
        return self.ev.batch

    @property
    def md_engine(self):
        return self.md.batch

    def footprint(self, req):
        s = req.system
        return self.ev.batch.footprint(s.N, len(s.exclusion_idxs), _terms(s, "bond_idxs"), _terms(s, "angle_idxs"))

    def bytes_in_use(self):
        return self.ev.batch.bytes_in_use() + self.md.batch.bytes_in_use()

    def submit(self, req):
        self.waiting.append(req)

    def _admit(self, kind, engine, now):
        """FIFO admission of arrived requests of one kind into an idle engine
        while the HBM budget allows (a request that does not fit blocks the
        later ones of its kind, keeping arrival order). MD segments are held
        to their share of the budget and to md_max_atoms resident atoms."""
        used = self.bytes_in_use()
        md_used = self.md.batch.bytes_in_use()
        md_atoms = sum(r.system.N for r in self.md.running)
        keep, blocked = [], False
        for req in self.waiting:
            if req.kind != kind or blocked or req.arrival > now:
                keep.append(req)
                continue
            need = self.footprint(req)
            if need > self.budget:
                raise RuntimeError(f"request {req.rid} needs {need} bytes, above the HBM budget")
            over = used + need > self.budget
            if kind == "md" and md_used > 0:  # an MD segment alone is always admissible
                over = over or md_used + need > self.md_budget or md_atoms + req.system.N > self.md_max_atoms
            if over:
                blocked = True
                keep.append(req)
                continue
            if kind == "md":
                md_used += need
                md_atoms += req.system.N
            if kind == "eval":
                req._replica = engine.batch.add(req.system, req.lam)
            else:
                req._replica = engine.batch.add(req.system, req.lam, v=req.v0, md=req.md, seed=req.seed)
            req.admitted = time.perf_counter()
            engine.running.append(req)
            used += need
        self.waiting = keep
        self.peak_bytes = max(self.peak_bytes, used)

    def _service_eval(self, now):
        e = self.ev
        if not e.idle():
            return False
        if e.running:  # the batch in flight has finished: answer it
            for req in e.running:
                req.result = e.batch.result_fixed(req._replica)
                req.finished = time.perf_counter()
                e.batch.remove(req._replica)
                self.done.append(req)
            e.running = []
            e.event = None
        self._admit("eval", e, now)
        if e.running:
            e.batch.evaluate()
            e.mark()
            return True
        return False

    def _service_md(self, now):
        e = self.md
        if not e.idle():
            return False
        if e.event is not None:  # the chunk in flight has finished
            still = []
            for req in e.running:
                req.steps_done += e.last_chunk
                if req.steps_done >= req.n_steps:
                    req.result = (e.batch.get_x(req._replica), e.batch.get_v(req._replica))
                    req.finished = time.perf_counter()
                    e.batch.remove(req._replica)
                    self.done.append(req)
                else:
                    still.append(req)
            e.running = still
            e.event = None
        self._admit("md", e, now)
        if e.running:
            n = min(self.md_chunk, min(r.n_steps - r.steps_done for r in e.running))
            e.batch.md(n, chunk=n, use_graph=self.md_graphs)
            e.last_chunk = n
            self.md_chunk_steps.append(n)
            e.mark()
            return True
        return False

    def step(self):
        """One pass of the loop: service each idle engine (collect, admit,
        launch). Returns True when something was launched."""
        now = time.perf_counter()
        a = self._service_eval(now)
        b = self._service_md(now)
        self.iterations += 1
        return a or b

    def busy(self):
        return bool(self.waiting or self.ev.running or self.md.running)

    def run(self, requests, t0=None, poll_s=2e-4):
        """Serves `requests` (arrival times in seconds relative to t0, default
        now) until all are done; returns them in completion order. A request's
        latency is finished - arrival (both absolute after this call)."""
        t0 = time.perf_counter() if t0 is None else t0
        for r in requests:
            r.arrival = t0 + r.arrival
            self.submit(r)
        while self.busy():
            launched = self.step()
            if not launched:
                # nothing to do until a launch completes or a request arrives
                now = time.perf_counter()
                nxt = min((r.arrival for r in self.waiting), default=now + poll_s)
                time.sleep(max(0.0, min(poll_s, nxt - now)))
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
