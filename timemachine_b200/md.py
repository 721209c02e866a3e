"""MD drivers of the nonbonded potential with timemachine's Python surface.

Mirrors timemachine/lib/__init__.py (LangevinIntegrator, MonteCarloBarostat
descriptors with .impl()) and custom_ops.Context
(timemachine/cpp/src/wrap_kernels.cpp Context binding: multiple_steps,
get_x_t, get_v_t, get_box, set_x_t). The step loop runs natively
(timemachine_b200/csrc/md.cu) with each step replayed as a CUDA graph.
"""

import ctypes

import numpy as np

from . import _lib

BOLTZ = 0.008314462618  # kJ/mol/K


def langevin_coefficients(temperature, dt, friction, masses):
    """timemachine/integrator.py:17-46: (ca, cb, cc) of BAOAB Langevin."""
    kT = BOLTZ * temperature
    nscale = np.sqrt(kT / masses)
    ca = np.exp(-friction * dt)
    cb = dt / masses
    cc = np.sqrt(1 - np.exp(-2 * friction * dt)) * nscale
    return ca, cb, cc


class LangevinIntegrator:
    """timemachine/lib/__init__.py:7-20 (cbs negated: forces are du_dx)."""

    def __init__(self, temperature, dt, friction, masses, seed):
        self.dt = dt
        self.seed = seed
        ca, cb, cc = langevin_coefficients(temperature, dt, friction, np.asarray(masses, dtype=np.float64))
        cb *= -1
        self.ca = ca
        self.cbs = cb
        self.ccs = cc

    def impl(self):
        return self


class MonteCarloBarostat:
    """timemachine/lib/__init__.py:23-38."""

    def __init__(self, N, pressure, temperature, group_idxs, interval, seed):
        self.N = N
        self.pressure = pressure
        self.temperature = temperature
        self.group_idxs = group_idxs
        self.interval = interval
        self.seed = seed
        self._contexts = []  # contexts driving this barostat (weak references)

    def impl(self, bound_potentials=None):
        return self

    def _live(self):
        out = []
        for ref in self._contexts:
            c = ref()
            if c is not None and getattr(c, "_h", None):
                out.append(c)
        return out

    def set_pressure(self, pressure):
        """custom_ops.MonteCarloBarostat.set_pressure (bar)."""
        self.pressure = pressure
        for c in self._live():
            _lib.check(c._lib.tmnb_context_barostat_set_pressure(c._h, float(pressure)))

    def set_interval(self, interval):
        """custom_ops.MonteCarloBarostat.set_interval: restarts the move counter."""
        self.interval = interval
        for c in self._live():
            _lib.check(c._lib.tmnb_context_barostat_set_interval(c._h, int(interval)))

    def get_interval(self):
        return self.interval

    def group_of(self):
        g = np.full(self.N, -1, dtype=np.int32)
        seen = set()
        for k, atoms in enumerate(self.group_idxs):
            for a in atoms:
                a = int(a)
                if a < 0 or a >= self.N:
                    raise RuntimeError("Grouped indices must be between 0 and N")
                if a in seen:
                    raise RuntimeError("All grouped indices must be unique")
                seen.add(a)
                g[a] = k
        return g


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class Context:
    """custom_ops.Context(x0, v0, box, integrator, bound_potentials, barostat=None)."""

    def __init__(self, x0, v0, box, integrator, bound_potentials, barostat=None, use_graphs=True):
        self._lib = _lib.lib()
        x0 = np.ascontiguousarray(x0, dtype=np.float64)
        v0 = np.ascontiguousarray(v0, dtype=np.float64)
        box = np.ascontiguousarray(box, dtype=np.float64)
        self.N = x0.shape[0]
        self.dt = integrator.dt
        self.use_graphs = use_graphs
        self._bps = list(bound_potentials)  # keep the potentials alive
        n = len(self._bps)
        handles = (ctypes.c_void_p * n)(*[bp.potential.handle for bp in self._bps])
        self._params = [np.ascontiguousarray(bp.params, dtype=np.float64).reshape(-1) for bp in self._bps]
        pptrs = (ctypes.c_void_p * n)(*[p.ctypes.data for p in self._params])
        sizes = (ctypes.c_int * n)(*[p.size for p in self._params])
        cbs = np.ascontiguousarray(integrator.cbs, dtype=np.float64)
        ccs = np.ascontiguousarray(integrator.ccs, dtype=np.float64)
        h = ctypes.c_void_p()
        _lib.check(
            self._lib.tmnb_context_create(
                self.N, _p(x0), _p(v0), _p(box), float(integrator.dt), float(integrator.ca), _p(cbs), _p(ccs),
                int(integrator.seed) & ((1 << 64) - 1), n, handles, pptrs, sizes, ctypes.byref(h),
            )
        )
        self._h = h
        if barostat is not None:
            import weakref

            barostat._contexts.append(weakref.ref(self))
            g = barostat.group_of()
            _lib.check(
                self._lib.tmnb_context_set_barostat(
                    self._h, float(barostat.pressure), float(barostat.temperature), _p(g), int(barostat.interval),
                    int(barostat.seed) & ((1 << 64) - 1),
                )
            )

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            try:
                self._lib.tmnb_context_destroy(h)
            except Exception:
                pass

    def multiple_steps(self, lambda_schedule, store_du_dl_interval=0, store_x_interval=0):
        """(du_dls, xs, boxes) as timemachine's Context.multiple_steps returns them."""
        lam = np.ascontiguousarray(np.atleast_1d(lambda_schedule), dtype=np.float64)
        n = lam.size
        n_dl = n // store_du_dl_interval if store_du_dl_interval > 0 else 0
        n_x = n // store_x_interval if store_x_interval > 0 else 0
        du_dl = np.zeros(n_dl)
        xs = np.zeros((n_x, self.N, 3))
        boxes = np.zeros((n_x, 3, 3))
        _lib.check(
            self._lib.tmnb_context_multiple_steps(
                self._h, n, _p(lam), int(store_du_dl_interval), _p(du_dl), int(store_x_interval), _p(xs), _p(boxes),
                1 if self.use_graphs else 0,
            )
        )
        return du_dl, xs, boxes

    def multiple_steps_U(self, lamb, n_steps, lambda_windows, store_u_interval, store_x_interval):
        """(U [F, K], xs, boxes): n_steps at lamb, the total energy at every
        lambda window every store_u_interval steps (timemachine/cpp/src/wrap_kernels.cpp:186-219;
        intervals <= 0 mean n_steps)."""
        windows = np.ascontiguousarray(np.atleast_1d(lambda_windows), dtype=np.float64)
        n_steps = int(n_steps)
        u_int = n_steps if store_u_interval <= 0 else int(store_u_interval)
        x_int = n_steps if store_x_interval <= 0 else int(store_x_interval)
        F_u = n_steps // u_int if u_int > 0 else 0
        F_x = n_steps // x_int if x_int > 0 else 0
        u = np.zeros((F_u, windows.size))
        xs = np.zeros((F_x, self.N, 3))
        boxes = np.zeros((F_x, 3, 3))
        _lib.check(
            self._lib.tmnb_context_multiple_steps_U(
                self._h, float(lamb), n_steps, windows.size, _p(windows), u_int, x_int, _p(u), _p(xs), _p(boxes),
                1 if self.use_graphs else 0,
            )
        )
        return u, xs, boxes

    def step(self, lamb):
        self.multiple_steps(np.array([lamb]))

    def _get(self, name, shape):
        out = np.zeros(shape)
        _lib.check(getattr(self._lib, "tmnb_context_" + name)(self._h, _p(out)))
        return out

    def get_x_t(self):
        return self._get("get_x", (self.N, 3))

    def get_v_t(self):
        return self._get("get_v", (self.N, 3))

    def get_box(self):
        return self._get("get_box", (3, 3))

    def set_x_t(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        _lib.check(self._lib.tmnb_context_set_x(self._h, _p(x)))

    def set_v_t(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        _lib.check(self._lib.tmnb_context_set_v(self._h, _p(v)))

    def set_box(self, box):
        box = np.ascontiguousarray(box, dtype=np.float64)
        _lib.check(self._lib.tmnb_context_set_box(self._h, _p(box)))

    def barostat_last_move(self):
        """The last barostat move: dict of rand0, rand1, proposal_scale,
        volume_delta, length_scale, accepted, volume_scale (after adaptation),
        pressure (kJ/mol/nm^3), u_before / u_after (fixed point, uint64)."""
        vals = np.zeros(8)
        us = np.zeros(2, dtype=np.uint64)
        _lib.check(self._lib.tmnb_context_barostat_last_move(self._h, _p(vals), _p(us)))
        keys = ["rand0", "rand1", "proposal_scale", "volume_delta", "length_scale", "accepted", "volume_scale",
                "pressure"]
        out = dict(zip(keys, vals.tolist()))
        out["accepted"] = bool(out["accepted"])
        out["u_before"], out["u_after"] = np.uint64(us[0]), np.uint64(us[1])
        return out

    def barostat_stats(self):
        a, t, vs = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_double()
        _lib.check(self._lib.tmnb_context_barostat_stats(self._h, ctypes.byref(a), ctypes.byref(t), ctypes.byref(vs)))
        return a.value, t.value, vs.value
