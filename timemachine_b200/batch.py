"""Replica batch: many systems x lambda windows evaluated and simulated together.

The reference runs replicas one at a time (one ``execute_selective`` / one
``Context`` per system and lambda window). ``ReplicaBatch`` holds any mix of
systems of different sizes, each replica at its own lambda, and serves all of
them with one launch sequence per step (timemachine_b200/csrc/batch.cu): a
single persistent pair kernel over every replica's tile work, and for MD a
CUDA graph per chunk of steps. Each replica's results equal a single-system
evaluation of the same inputs bit for bit, whatever else is in the batch.

``autotune`` picks the tile schedule (tiles per work item, neighbour-list
padding, Hilbert grid resolution, pair-kernel CTAs per SM) by timing the
batch's own workload.
"""

import ctypes
import itertools
import time

import numpy as np

from . import _lib
from .fixed_point import du_dp_fixed_to_float, fixed_to_float, sum_fixed
from .md import langevin_coefficients

_X, _V, _BOX, _DU_DX, _DU_DP, _DU_DL, _U = range(7)


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dtype):
    return None if a is None else np.ascontiguousarray(a, dtype=dtype)


def _terms(system, name, width):
    a = getattr(system, name, None)
    return np.zeros((0, width)) if a is None else np.asarray(a).reshape(-1, width)


class ReplicaBatch:
    def __init__(self, priority=None):
        """priority: CUDA stream priority of the batch's stream (lower numbers
        first; None: the default priority)."""
        self._lib = _lib.lib()
        h = ctypes.c_void_p()
        _lib.check(self._lib.tmnb_batch_create(ctypes.byref(h)))
        self._h = h
        if priority is not None:
            _lib.check(self._lib.tmnb_batch_set_priority(self._h, int(priority)))
        self._n = {}
        self.tuning = {"chunk": 4, "padding": 0.1, "grid_bits_offset": 0, "pair_ctas_per_sm": 0, "rows": 16}

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            try:
                self._lib.tmnb_batch_destroy(h)
            except Exception:
                pass

    def __len__(self):
        return self._lib.tmnb_batch_size(self._h)

    # -- membership ------------------------------------------------------------
    def add(self, system, lam, x=None, v=None, box=None, md=None, seed=0):
        """Adds one replica of `system` (a testsystems.System-like object with x,
        box, params, exclusion_idxs, scales, lambda_plane_idxs,
        lambda_offset_idxs, beta, cutoff and optional bond/angle terms) at
        lambda `lam`. md: None, or dict(temperature, dt, friction) with the
        system's masses, for Langevin MD. Returns the replica id."""
        N = system.x.shape[0]
        x = _c(system.x if x is None else x, np.float64)
        box = _c(system.box if box is None else box, np.float64)
        v = _c(v, np.float64)
        params = _c(system.params, np.float64)
        plane = _c(system.lambda_plane_idxs, np.int32)
        offset = _c(system.lambda_offset_idxs, np.int32)
        excl = _c(np.asarray(system.exclusion_idxs).reshape(-1, 2), np.int32)
        scales = _c(np.asarray(system.scales).reshape(-1, 2), np.float64)
        bonds = _c(_terms(system, "bond_idxs", 2), np.int32)
        bparams = _c(_terms(system, "bond_params", 2), np.float64)
        angles = _c(_terms(system, "angle_idxs", 3), np.int32)
        aparams = _c(_terms(system, "angle_params", 2), np.float64)
        ca, dt, cbs, ccs = 0.0, 0.0, None, None
        if md is not None:
            ca, cb, cc = langevin_coefficients(md["temperature"], md["dt"], md["friction"], np.asarray(system.masses))
            cbs = _c(-cb, np.float64)
            ccs = _c(cc, np.float64)
            dt = float(md["dt"])

        def opt(a):
            return _p(a) if a.size else None

        rid = ctypes.c_int32()
        _lib.check(
            self._lib.tmnb_batch_add(
                self._h, N, _p(x), _p(v), _p(box), _p(params), _p(plane), _p(offset),
                excl.shape[0], opt(excl), opt(scales),
                bonds.shape[0], opt(bonds), opt(bparams),
                angles.shape[0], opt(angles), opt(aparams),
                float(system.beta), float(system.cutoff), float(lam), dt, float(ca), _p(cbs), _p(ccs),
                int(seed) & ((1 << 64) - 1), ctypes.byref(rid),
            )
        )
        self._n[rid.value] = N
        return rid.value

    def remove(self, rid):
        _lib.check(self._lib.tmnb_batch_remove(self._h, int(rid)))
        self._n.pop(rid, None)

    def footprint(self, N, M=0, B=0, A=0):
        """Device bytes one replica of N atoms (M exclusions, B bonds, A angles) holds."""
        b = ctypes.c_ulonglong()
        _lib.check(self._lib.tmnb_batch_footprint(self._h, int(N), int(M), int(B), int(A), ctypes.byref(b)))
        return b.value

    def bytes_in_use(self):
        b = ctypes.c_ulonglong()
        _lib.check(self._lib.tmnb_batch_bytes_in_use(self._h, ctypes.byref(b)))
        return b.value

    def ids(self):
        return sorted(self._n)

    # -- work ------------------------------------------------------------------
    def set_tuning(self, chunk=4, padding=0.1, grid_bits_offset=0, pair_ctas_per_sm=0, rows=16):
        """Schedule of every replica: tiles per work item, neighbour-list
        padding, Hilbert grid offset, pair-kernel CTAs per SM (0: occupancy)
        and rows per tile (32, 16 or 8). Results do not depend on it."""
        if rows != self.tuning.get("rows", 16):
            _lib.check(self._lib.tmnb_batch_set_tile_rows(self._h, int(rows)))
        _lib.check(
            self._lib.tmnb_batch_set_tuning(self._h, int(chunk), float(padding), int(grid_bits_offset), int(pair_ctas_per_sm))
        )
        self.tuning = {
            "chunk": chunk, "padding": padding, "grid_bits_offset": grid_bits_offset, "pair_ctas_per_sm": pair_ctas_per_sm,
            "rows": rows,
        }

    def evaluate(self, du_dx=True, du_dp=True, du_dl=True, u=True):
        """One evaluation of every replica (asynchronous; results via result())."""
        _lib.check(self._lib.tmnb_batch_evaluate(self._h, int(du_dx), int(du_dp), int(du_dl), int(u)))

    def md(self, n_steps, chunk=500, use_graph=True):
        """n_steps Langevin steps of every replica (asynchronous)."""
        _lib.check(self._lib.tmnb_batch_md(self._h, int(n_steps), int(chunk), int(use_graph)))

    @property
    def stream(self):
        """The batch's cudaStream_t (int); every batch call is ordered on it."""
        s = ctypes.c_void_p()
        _lib.check(self._lib.tmnb_batch_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def synchronize(self):
        _lib.check(self._lib.tmnb_batch_synchronize(self._h))

    # -- state -----------------------------------------------------------------
    def _get(self, rid, which, shape, dtype):
        out = np.zeros(shape, dtype=dtype)
        _lib.check(self._lib.tmnb_batch_get(self._h, int(rid), which, _p(out)))
        return out

    def _size(self, rid):
        if rid not in self._n:
            raise RuntimeError(f"unknown replica id {rid}")
        return self._n[rid]

    def get_x(self, rid):
        return self._get(rid, _X, (self._size(rid), 3), np.float64)

    def get_v(self, rid):
        return self._get(rid, _V, (self._size(rid), 3), np.float64)

    def get_box(self, rid):
        return self._get(rid, _BOX, (3, 3), np.float64)

    def set_x(self, rid, x):
        x = _c(x, np.float64)
        _lib.check(self._lib.tmnb_batch_set(self._h, int(rid), _X, _p(x)))

    def set_v(self, rid, v):
        v = _c(v, np.float64)
        _lib.check(self._lib.tmnb_batch_set(self._h, int(rid), _V, _p(v)))

    def result_fixed(self, rid):
        """Raw int64 fixed-point outputs of the last evaluation: du_dx [N,3], du_dp [N,3], du_dl [N], u [N]."""
        N = self._size(rid)
        return (
            self._get(rid, _DU_DX, (N, 3), np.uint64),
            self._get(rid, _DU_DP, (N, 3), np.uint64),
            self._get(rid, _DU_DL, (N,), np.uint64),
            self._get(rid, _U, (N,), np.uint64),
        )

    def result(self, rid):
        """(du_dx, du_dp, du_dl, u) of the last evaluation, decoded as the reference decodes them."""
        dx, dp, dl, u = self.result_fixed(rid)
        return fixed_to_float(dx), du_dp_fixed_to_float(dp), fixed_to_float(sum_fixed(dl)), fixed_to_float(sum_fixed(u))

    def error(self, rid):
        c = ctypes.c_int32()
        _lib.check(self._lib.tmnb_batch_error(self._h, int(rid), ctypes.byref(c)))
        return c.value

    def stats(self, rid):
        t, i, r = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        _lib.check(self._lib.tmnb_batch_stats(self._h, int(rid), ctypes.byref(t), ctypes.byref(i), ctypes.byref(r)))
        return t.value, i.value, r.value

    # -- schedule autotuner ----------------------------------------------------
    def autotune(self, mode="md", steps=20, repeats=2, candidates=None, chunk=None):
        """Times the batch's own workload under each candidate schedule and keeps
        the fastest. mode "md": `steps` Langevin steps (rebuild cadence
        included; the replicas' states advance); "eval": `steps` evaluations.
        Candidates: dicts of set_tuning keywords (default: tiles per item
        {1, 2, 4, 8} x padding {0.06, 0.1, 0.14} x Hilbert grid offset {0, 1}).
        Returns (best, [(config, seconds), ...])."""
        if candidates is None:
            candidates = [
                {"chunk": c, "padding": p, "grid_bits_offset": g, "pair_ctas_per_sm": 0}
                for c, p, g in itertools.product([1, 2, 4, 8], [0.06, 0.1, 0.14], [0, 1])
            ]

        def run():
            if mode == "md":
                self.md(steps, chunk=chunk or steps, use_graph=True)
            else:
                for _ in range(steps):
                    self.evaluate()

        timings = []
        for cfg in candidates:
            self.set_tuning(**cfg)
            run()  # warm-up: rebuild + graph capture
            self.synchronize()
            best = float("inf")
            for _ in range(repeats):
                t0 = time.perf_counter()
                run()
                self.synchronize()
                best = min(best, time.perf_counter() - t0)
            timings.append((dict(cfg), best))
        best_cfg = min(timings, key=lambda t: t[1])[0]
        self.set_tuning(**best_cfg)
        return best_cfg, timings
