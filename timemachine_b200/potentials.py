"""Nonbonded potentials with timemachine's Python surface, on the B200 kernels.

Mirrors timemachine/lib/potentials.py (classes, constructor arguments,
bind/unbound_impl/bound_impl) and the methods that
timemachine/cpp/src/wrap_kernels.cpp:334-723 binds on the implementation
objects (execute, execute_selective, execute_selective_batch, execute_du_dx,
BoundPotential.execute / execute_fixed, disable_hilbert_sort,
set_nblist_padding). Results are float64 numpy arrays decoded from the
int64 fixed-point accumulators exactly as the reference decodes them.

Device-resident use goes through ``Potential.execute_device`` on torch CUDA
tensors (no host copies, no host synchronisation).
"""

import ctypes
import itertools

import numpy as np

from . import _lib
from .fixed_point import FIXED_EXPONENT, fixed_to_float, sum_fixed

__all__ = [
    "CustomOpWrapper",
    "Nonbonded",
    "NonbondedInterpolated",
    "NonbondedAllPairs",
    "NonbondedAllPairsInterpolated",
    "NonbondedInteractionGroup",
    "NonbondedInteractionGroupInterpolated",
    "NonbondedPairList",
    "NonbondedPairListNegated",
    "NonbondedPairListInterpolated",
    "NonbondedPairListNegatedInterpolated",
    "Potential",
    "BoundPotential",
]


def _ptr(a):
    """Address of a contiguous numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.c_void_p)


def _precision_bits(precision):
    """np.float32 -> 32 (FP32 pair arithmetic, the reference's _f32 kernels);
    np.float64 -> 64 (FP64 pair arithmetic, the reference's _f64 kernels)."""
    if precision == np.float64:
        return 64
    if precision == np.float32:
        return 32
    raise RuntimeError(f"unsupported precision {precision!r}: use np.float32 or np.float64")


_TRANSFORM_NAMES = ("transform_lambda_charge", "transform_lambda_sigma", "transform_lambda_epsilon", "transform_lambda_w")


def _transforms(extra):
    """The four lambda-transform expressions that follow a constructor's
    regular arguments (timemachine/cpp/src/wrap_kernels.cpp:843-893), "lambda"
    where absent."""
    extra = list(extra)
    if len(extra) > 4:
        raise RuntimeError(f"expected at most 4 lambda transform expressions, got {len(extra)}")
    out = []
    for k, name in enumerate(_TRANSFORM_NAMES):
        v = extra[k] if k < len(extra) else "lambda"
        if not isinstance(v, str):
            raise RuntimeError(f"{name} must be a string expression in lambda, got {v!r}")
        out.append(v)
    return out


def _apply_transforms(handle, extra):
    t = _transforms(extra)
    if any(e.strip() != "lambda" for e in t):
        _lib.check(_lib.lib().tmnb_potential_set_lambda_transforms(handle, *[e.encode() for e in t]))


def lambda_transform(expression, lam):
    """(f, df/dlambda) of one lambda-transform expression at lam, as the
    potentials evaluate their schedules (host-side parser of the C ABI)."""
    f, df = ctypes.c_double(), ctypes.c_double()
    _lib.check(_lib.lib().tmnb_lambda_transform_eval(str(expression).encode(), float(lam), ctypes.byref(f),
                                                     ctypes.byref(df)))
    return f.value, df.value


class Potential:
    """Unbound implementation: one native handle (the reference's custom_ops.Potential)."""

    def __init__(self, handle, name, interpolated):
        self._h = handle
        self._name = name
        self.interpolated = interpolated
        self._lib = _lib.lib()

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            try:
                self._lib.tmnb_potential_destroy(h)
            except Exception:
                pass

    @property
    def handle(self):
        return self._h

    # -- configuration (timemachine/cpp/src/nonbonded_all_pairs.cu:180-187) --
    def set_nblist_padding(self, padding):
        _lib.check(self._lib.tmnb_potential_set_nblist_padding(self._h, float(padding)))

    def disable_hilbert_sort(self):
        _lib.check(self._lib.tmnb_potential_disable_hilbert_sort(self._h))

    def set_tile_rows(self, rows=16):
        """Rows per neighbour-list tile: 16 (default), 32 or 8 slots (identical
        results; FP64 potentials use 16)."""
        _lib.check(self._lib.tmnb_potential_set_tile_rows(self._h, int(rows)))

    def num_params(self):
        return self._lib.tmnb_potential_num_params(self._h)

    def num_atoms(self):
        return self._lib.tmnb_potential_num_atoms(self._h)

    # -- host entry points ---------------------------------------------------
    def _execute_fixed(self, coords, params, box, lam, du_dx, du_dp, du_dl, u):
        coords = np.ascontiguousarray(coords, dtype=np.float64)
        params = np.ascontiguousarray(params, dtype=np.float64)
        box = np.ascontiguousarray(box, dtype=np.float64)
        if coords.ndim != 2 or coords.shape[1] != 3:
            raise RuntimeError("coords must have shape (N, 3)")
        if box.size != 9:
            raise RuntimeError("box must have shape (3, 3)")
        N = coords.shape[0]
        P = params.size
        out_dx = np.empty((N, 3), dtype=np.uint64) if du_dx else None
        out_dp = np.empty(P, dtype=np.uint64) if du_dp else None
        out_dl = np.empty(N, dtype=np.uint64) if du_dl else None
        out_u = np.empty(N, dtype=np.uint64) if u else None
        _lib.check(
            self._lib.tmnb_potential_execute_host(
                self._h,
                N,
                P,
                _ptr(coords),
                _ptr(params),
                _ptr(box),
                float(lam),
                _ptr(out_dx),
                _ptr(out_dp),
                _ptr(out_dl),
                _ptr(out_u),
            )
        )
        return out_dx, out_dp, out_dl, out_u

    def _decode_dp(self, fixed):
        """Fixed-point du_dp to float with this potential's per-column exponents
        (Potential::du_dp_fixed_to_float, timemachine/cpp/src/potential.hpp:64)."""
        fixed = np.ascontiguousarray(fixed, dtype=np.uint64)
        flat = fixed.reshape(-1, fixed.shape[-1]) if fixed.ndim > 1 else fixed.reshape(1, -1)
        out = np.empty(flat.shape, dtype=np.float64)
        for r in range(flat.shape[0]):
            row = np.ascontiguousarray(flat[r])
            _lib.check(
                self._lib.tmnb_potential_du_dp_fixed_to_float(
                    self._h, self.num_atoms(), row.size, _ptr(row), _ptr(out[r])
                )
            )
        return out.reshape(fixed.shape)

    def execute_selective(self, coords, params, box, lam, compute_du_dx, compute_du_dp, compute_du_dl, compute_u):
        """timemachine/cpp/src/wrap_kernels.cpp:552-625: tuple with None for outputs not requested."""
        params = np.asarray(params, dtype=np.float64)
        fdx, fdp, fdl, fu = self._execute_fixed(
            coords, params, box, lam, compute_du_dx, compute_du_dp, compute_du_dl, compute_u
        )
        du_dx = fixed_to_float(fdx) if compute_du_dx else None
        du_dp = self._decode_dp(fdp).reshape(params.shape) if compute_du_dp else None
        du_dl = fixed_to_float(sum_fixed(fdl)) if compute_du_dl else None
        u = fixed_to_float(sum_fixed(fu)) if compute_u else None
        return du_dx, du_dp, du_dl, u

    def execute(self, coords, params, box, lam):
        """timemachine/cpp/src/wrap_kernels.cpp:339-380: (du_dx, du_dp, du_dl, u)."""
        return self.execute_selective(coords, params, box, lam, True, True, True, True)

    def execute_du_dx(self, coords, params, box, lam):
        """timemachine/cpp/src/wrap_kernels.cpp:626-651."""
        return self.execute_selective(coords, params, box, lam, True, False, False, False)[0]

    def execute_selective_batch(
        self, coords, params, boxes, lambdas, compute_du_dx, compute_du_dp, compute_du_dl, compute_u
    ):
        """timemachine/cpp/src/wrap_kernels.cpp:381-551: every (coords, params, lambda) combination."""
        coords = np.ascontiguousarray(coords, dtype=np.float64)
        params = np.ascontiguousarray(params, dtype=np.float64)
        boxes = np.ascontiguousarray(boxes, dtype=np.float64)
        lambdas = np.ascontiguousarray(np.atleast_1d(lambdas), dtype=np.float64)
        if coords.ndim != 3 and boxes.ndim != 3:
            raise RuntimeError("coords and boxes must have 3 dimensions")
        if coords.shape[0] != boxes.shape[0]:
            raise RuntimeError("number of batches of coords and boxes don't match")
        if params.ndim < 2:
            raise RuntimeError("parameters must have at least 2 dimensions")
        if lambdas.size < 1:
            raise RuntimeError("lambdas must have at least 1 value")
        C, N, _ = coords.shape
        Pb = params.shape[0]
        P = params.size // Pb
        L = lambdas.size
        E = C * Pb * L
        out_dx = np.empty((E, N, 3), dtype=np.uint64) if compute_du_dx else None
        out_dp = np.empty((E, P), dtype=np.uint64) if compute_du_dp else None
        out_dl = np.empty((E, N), dtype=np.uint64) if compute_du_dl else None
        out_u = np.empty((E, N), dtype=np.uint64) if compute_u else None
        _lib.check(
            self._lib.tmnb_potential_execute_batch_host(
                self._h,
                C,
                N,
                Pb,
                P,
                L,
                _ptr(coords),
                _ptr(params),
                _ptr(boxes),
                _ptr(lambdas),
                _ptr(out_dx),
                _ptr(out_dp),
                _ptr(out_dl),
                _ptr(out_u),
            )
        )
        res = [None, None, None, None]
        if compute_du_dx:
            res[0] = fixed_to_float(out_dx).reshape(C, Pb, L, N, 3)
        if compute_du_dp:
            res[1] = self._decode_dp(out_dp).reshape((C, Pb, L) + params.shape[1:])
        if compute_du_dl:
            res[2] = np.array([fixed_to_float(sum_fixed(r)) for r in out_dl]).reshape(C, Pb, L)
        if compute_u:
            res[3] = np.array([fixed_to_float(sum_fixed(r)) for r in out_u]).reshape(C, Pb, L)
        return tuple(res)

    def du_dp_fixed_to_float(self, N, P, du_dp):
        return self._decode_dp(np.asarray(du_dp, dtype=np.uint64).reshape(-1))

    def execute_windows_fixed(self, coords, params, box, lambdas, du_dx=True, du_dp=True, du_dl=True, u=True):
        """K lambda windows of one (coords, params, box) in one multi-window
        evaluation: raw uint64 fixed-point outputs with leading axis K (None
        where not requested). Each window equals execute at lambdas[k] bit for bit."""
        coords = np.ascontiguousarray(coords, dtype=np.float64)
        params = np.ascontiguousarray(params, dtype=np.float64)
        box = np.ascontiguousarray(box, dtype=np.float64)
        lambdas = np.ascontiguousarray(np.atleast_1d(lambdas), dtype=np.float64)
        if coords.ndim != 2 or coords.shape[1] != 3:
            raise RuntimeError("coords must have shape (N, 3)")
        if box.size != 9:
            raise RuntimeError("box must have shape (3, 3)")
        N, P, K = coords.shape[0], params.size, lambdas.size
        out_dx = np.empty((K, N, 3), dtype=np.uint64) if du_dx else None
        out_dp = np.empty((K, P), dtype=np.uint64) if du_dp else None
        out_dl = np.empty((K, N), dtype=np.uint64) if du_dl else None
        out_u = np.empty((K, N), dtype=np.uint64) if u else None
        _lib.check(
            self._lib.tmnb_potential_execute_windows_host(
                self._h,
                N,
                P,
                _ptr(coords),
                _ptr(params),
                _ptr(box),
                K,
                _ptr(lambdas),
                _ptr(out_dx),
                _ptr(out_dp),
                _ptr(out_dl),
                _ptr(out_u),
            )
        )
        return out_dx, out_dp, out_dl, out_u

    def execute_windows(self, coords, params, box, lambdas):
        """(du_dx [K,N,3], du_dp [K,*params.shape], du_dl [K], u [K]) for K lambda windows."""
        params = np.asarray(params, dtype=np.float64)
        fdx, fdp, fdl, fu = self.execute_windows_fixed(coords, params, box, lambdas)
        K = fdx.shape[0]
        du_dp = self._decode_dp(fdp).reshape((K,) + params.shape)
        du_dl = np.array([fixed_to_float(sum_fixed(r)) for r in fdl])
        u = np.array([fixed_to_float(sum_fixed(r)) for r in fu])
        return fixed_to_float(fdx), du_dp, du_dl, u

    # -- device entry point (torch tensors) -----------------------------------
    def execute_device(self, x, p, box, lam, du_dx=None, du_dp=None, du_dl=None, u=None, stream=None):
        """Accumulate into int64 device tensors (the C-ABI device contract).

        x [N,3] f64, p [P] f64, box [3,3] f64 on the same CUDA device; outputs are
        int64 tensors that the caller zeroes. ``stream``: torch.cuda.Stream, a raw
        cudaStream_t (int), or None for torch's current stream.
        """
        import torch

        def addr(t):
            if t is None:
                return None
            if not t.is_contiguous():
                raise RuntimeError("device tensors must be contiguous")
            return ctypes.c_void_p(t.data_ptr())

        if stream is None:
            stream = torch.cuda.current_stream(x.device).cuda_stream
        elif hasattr(stream, "cuda_stream"):
            stream = stream.cuda_stream
        _lib.check(
            self._lib.tmnb_potential_execute_device(
                self._h,
                x.shape[0],
                p.numel(),
                addr(x),
                addr(p),
                addr(box),
                float(lam),
                addr(du_dx),
                addr(du_dp),
                addr(du_dl),
                addr(u),
                ctypes.c_void_p(stream),
            )
        )

    def execute_windows_device(self, x, p, box, lambdas, du_dx=None, du_dp=None, du_dl=None, u=None, stream=None):
        """K lambda windows on device tensors; outputs [K,N,3] / [K,P] / [K,N]
        int64 tensors that accumulate (the caller zeroes them)."""
        import torch

        def addr(t):
            if t is None:
                return None
            if not t.is_contiguous():
                raise RuntimeError("device tensors must be contiguous")
            return ctypes.c_void_p(t.data_ptr())

        lam = np.ascontiguousarray(np.atleast_1d(lambdas), dtype=np.float64)
        if stream is None:
            stream = torch.cuda.current_stream(x.device).cuda_stream
        elif hasattr(stream, "cuda_stream"):
            stream = stream.cuda_stream
        _lib.check(
            self._lib.tmnb_potential_execute_windows_device(
                self._h,
                x.shape[0],
                p.numel(),
                addr(x),
                addr(p),
                addr(box),
                lam.size,
                _ptr(lam),
                addr(du_dx),
                addr(du_dp),
                addr(du_dl),
                addr(u),
                ctypes.c_void_p(stream),
            )
        )

    def adjoint_device(self, x, p, box, lam, g_du_dx, g_du_dl, grad_p, grad_w, stream=None):
        """Adds the vector-Jacobian product of (du_dx, du_dl) with upstream
        (g_du_dx [N,3] float64, g_du_dl float) into grad_p [P] and grad_w [N]
        (float64 device tensors): d/d params and d/d per-atom lambda offsets."""
        import torch

        def addr(t):
            if not t.is_contiguous():
                raise RuntimeError("device tensors must be contiguous")
            return ctypes.c_void_p(t.data_ptr())

        if stream is None:
            stream = torch.cuda.current_stream(x.device).cuda_stream
        elif hasattr(stream, "cuda_stream"):
            stream = stream.cuda_stream
        _lib.check(
            self._lib.tmnb_potential_adjoint_device(
                self._h, x.shape[0], p.numel(), addr(x), addr(p), addr(box), float(lam), addr(g_du_dx),
                float(g_du_dl), addr(grad_p), addr(grad_w), ctypes.c_void_p(stream),
            )
        )

    def check_device_error(self, stream=None):
        import torch

        if stream is None:
            stream = torch.cuda.current_stream().cuda_stream
        elif hasattr(stream, "cuda_stream"):
            stream = stream.cuda_stream
        _lib.check(self._lib.tmnb_potential_check_device_error(self._h, ctypes.c_void_p(stream)))

    def get_nblist(self, stream=None):
        """(perm [S] slot -> atom, tiles, rows) of the last rebuild; tiles[g] is
        an array of the column SLOTS (map them to atoms through perm) listed for
        row group g, whose rows are slots g*rows .. g*rows+rows-1."""
        S, G, cap = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_longlong()
        _lib.check(self._lib.tmnb_potential_nblist_shape(self._h, ctypes.byref(S), ctypes.byref(G), ctypes.byref(cap)))
        rows, CB = ctypes.c_int32(), ctypes.c_int32()
        _lib.check(self._lib.tmnb_potential_nblist_rows(self._h, ctypes.byref(rows), ctypes.byref(CB)))
        perm = np.zeros(S.value, dtype=np.uint32)
        nt = np.zeros(G.value, dtype=np.int32)
        cols = np.zeros(cap.value * 32, dtype=np.uint32)
        s = 0
        if stream is not None:
            s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        _lib.check(self._lib.tmnb_potential_copy_nblist(self._h, ctypes.c_void_p(s), _ptr(perm), _ptr(nt), _ptr(cols)))
        R, cb = rows.value, CB.value
        m = 32 // R
        nr = getattr(self, "_group_rows", None)
        tiles = []
        for g in range(G.value):
            if nr is None:
                # upper triangle: group g reaches the column blocks from b = g*R/32 on
                b = g // m
                off = m * (b * cb - (b * (b - 1)) // 2) + (g - b * m) * (cb - b)
            else:
                off = g * (cb - nr // 32)
            c = cols[off * 32 : (off + nt[g]) * 32]
            tiles.append(c[c < S.value])
        return perm, tiles, R

    def nblist_stats(self, stream=None):
        """(tiles, work items, rebuilds) of the last neighbour-list build (synchronises)."""
        t, i, r = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        s = 0
        if stream is not None:
            s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        _lib.check(
            self._lib.tmnb_potential_nblist_stats(
                self._h, ctypes.c_void_p(s), ctypes.byref(t), ctypes.byref(i), ctypes.byref(r)
            )
        )
        return t.value, i.value, r.value


class BoundPotential:
    """timemachine/cpp/src/bound_potential.cu + wrap_kernels.cpp:654-723."""

    def __init__(self, potential, params):
        self.potential = potential
        self.params = np.ascontiguousarray(params, dtype=np.float64)

    def get_potential(self):
        return self.potential

    def size(self):
        return self.params.size

    def execute(self, coords, box, lam):
        du_dx, _, du_dl, u = self.potential.execute_selective(coords, self.params, box, lam, True, False, True, True)
        return du_dx, du_dl, u

    def execute_fixed(self, coords, box, lam):
        _, _, _, fu = self.potential._execute_fixed(coords, self.params, box, lam, True, False, True, True)
        return np.array([sum_fixed(fu)], dtype=np.uint64)


class CustomOpWrapper:
    """timemachine/lib/potentials.py:13-39."""

    def __init__(self, *args):
        self.args = list(args)
        self.params = None

    def bind(self, params):
        self.params = params
        return self

    def unbound_impl(self, precision):
        raise NotImplementedError

    def bound_impl(self, precision):
        if self.params is None:
            raise ValueError("This op has not been bound to parameters.")
        return BoundPotential(self.unbound_impl(precision), self.params)


def _check_precision(precision):
    return _precision_bits(precision)


def _plane_offset(plane, offset):
    plane = np.ascontiguousarray(plane, dtype=np.int32)
    offset = np.ascontiguousarray(offset, dtype=np.int32)
    if plane.shape != offset.shape:
        raise RuntimeError("lambda offset idxs and plane idxs need to be equivalent")
    return plane, offset


def _pairs_scales(pair_idxs, scales):
    pair_idxs = np.ascontiguousarray(pair_idxs, dtype=np.int32)
    scales = np.ascontiguousarray(scales, dtype=np.float64)
    if pair_idxs.size % 2 != 0:
        raise RuntimeError(f"pair_idxs.size() must be even, but got {pair_idxs.size}")
    M = pair_idxs.size // 2
    if scales.size // 2 != M:
        raise RuntimeError(f"expected same number of pairs and scale tuples, but got {M} != {scales.size // 2}")
    return pair_idxs.reshape(-1, 2), scales.reshape(-1, 2), M


class NonbondedAllPairs(CustomOpWrapper):
    """args: (lambda_plane_idxs, lambda_offset_idxs, beta, cutoff[, atom_idxs])."""

    _interpolated = False

    def unbound_impl(self, precision):
        bits = _check_precision(precision)
        plane, offset = _plane_offset(self.args[0], self.args[1])
        beta, cutoff = float(self.args[2]), float(self.args[3])
        atom_idxs = self.args[4] if len(self.args) > 4 else None
        extra = self.args[5:]
        N = plane.size
        aidx, K = None, 0
        if atom_idxs is not None:
            aidx = np.ascontiguousarray(atom_idxs, dtype=np.int32)
            K = aidx.size
            if len(set(aidx.tolist())) != K:
                raise RuntimeError("atom indices must be unique")
        h = ctypes.c_void_p()
        lib = _lib.lib()
        _lib.check(
            lib.tmnb_all_pairs_create(
                N,
                _ptr(plane),
                _ptr(offset),
                beta,
                cutoff,
                _ptr(aidx),
                K,
                1 if self._interpolated else 0,
                bits,
                ctypes.byref(h),
            )
        )
        pot = Potential(h, "NonbondedAllPairs", self._interpolated)
        _apply_transforms(h, extra)
        return pot


class NonbondedAllPairsInterpolated(NonbondedAllPairs):
    _interpolated = True


class NonbondedInteractionGroup(CustomOpWrapper):
    """timemachine/lib/potentials.py:389-399: pairs of one row atom and one
    other atom. args: (row_atom_idxs, lambda_plane_idxs, lambda_offset_idxs, beta, cutoff
    [, 4 lambda transform expressions])."""

    _interpolated = False

    def unbound_impl(self, precision):
        bits = _check_precision(precision)
        rows = np.ascontiguousarray(self.args[0], dtype=np.int32).reshape(-1)
        if len(set(rows.tolist())) != rows.size:
            # the binding's unique_idxs (timemachine/cpp/src/wrap_kernels.cpp:922)
            raise RuntimeError("atom indices must be unique")
        plane, offset = _plane_offset(self.args[1], self.args[2])
        h = ctypes.c_void_p()
        lib = _lib.lib()
        _lib.check(
            lib.tmnb_interaction_group_create(
                plane.size,
                _ptr(rows) if rows.size else None,
                rows.size,
                _ptr(plane),
                _ptr(offset),
                float(self.args[3]),
                float(self.args[4]),
                1 if self._interpolated else 0,
                bits,
                ctypes.byref(h),
            )
        )
        pot = Potential(h, "NonbondedInteractionGroup", self._interpolated)
        _apply_transforms(h, self.args[5:])
        pot._group_rows = rows.size
        return pot


class NonbondedInteractionGroupInterpolated(NonbondedInteractionGroup):
    _interpolated = True


class NonbondedPairList(CustomOpWrapper):
    """args: (pair_idxs, scales, lambda_plane_idxs, lambda_offset_idxs, beta, cutoff
    [, 4 lambda transform expressions])."""

    _interpolated = False
    _negated = False

    def unbound_impl(self, precision):
        bits = _check_precision(precision)
        pairs, scales, M = _pairs_scales(self.args[0], self.args[1])
        plane, offset = _plane_offset(self.args[2], self.args[3])
        h = ctypes.c_void_p()
        lib = _lib.lib()
        _lib.check(
            lib.tmnb_pair_list_create(
                plane.size,
                _ptr(pairs),
                _ptr(scales),
                M,
                _ptr(plane),
                _ptr(offset),
                float(self.args[4]),
                float(self.args[5]),
                1 if self._negated else 0,
                1 if self._interpolated else 0,
                bits,
                ctypes.byref(h),
            )
        )
        pot = Potential(h, "NonbondedPairList", self._interpolated)
        _apply_transforms(h, self.args[6:])
        return pot


class NonbondedPairListNegated(NonbondedPairList):
    _negated = True


class NonbondedPairListInterpolated(NonbondedPairList):
    _interpolated = True


class NonbondedPairListNegatedInterpolated(NonbondedPairList):
    _negated = True
    _interpolated = True


class Nonbonded(CustomOpWrapper):
    """timemachine/lib/potentials.py:269-344.

    args: (exclusion_idxs, scale_factors, lambda_plane_idxs, lambda_offset_idxs, beta, cutoff
    [, 4 lambda transform expressions: NonbondedInterpolated only])

    The reference's Nonbonded.unbound_impl does not pass args[6:] on to its
    parts (timemachine/lib/potentials.py:284-301), so a non-identity
    expression there would be dropped without notice: this class raises
    instead. NonbondedInterpolated forwards them, as the reference's does
    (timemachine/lib/potentials.py:355,365).
    """

    _interpolated = False

    def __init__(self, *args):
        exclusion_idxs = np.asarray(args[0])
        exclusion_set = set()
        for src, dst in exclusion_idxs.reshape(-1, 2).tolist():
            src, dst = sorted((src, dst))
            exclusion_set.add((src, dst))
        assert len(exclusion_set) == exclusion_idxs.reshape(-1, 2).shape[0]
        super().__init__(*args)

    def unbound_impl(self, precision):
        bits = _check_precision(precision)
        extra = _transforms(self.args[6:])
        if not self._interpolated and any(e.strip() != "lambda" for e in extra):
            raise RuntimeError(
                "Nonbonded does not apply lambda transform expressions (the reference drops args[6:] here); "
                "use NonbondedInterpolated, NonbondedAllPairs or NonbondedPairList to apply them"
            )
        pairs, scales, M = _pairs_scales(self.get_exclusion_idxs(), self.get_scale_factors())
        plane, offset = _plane_offset(self.get_lambda_plane_idxs(), self.get_lambda_offset_idxs())
        h = ctypes.c_void_p()
        lib = _lib.lib()
        _lib.check(
            lib.tmnb_nonbonded_create(
                plane.size,
                _ptr(pairs),
                _ptr(scales),
                M,
                _ptr(plane),
                _ptr(offset),
                float(self.get_beta()),
                float(self.get_cutoff()),
                1 if self._interpolated else 0,
                bits,
                ctypes.byref(h),
            )
        )
        pot = Potential(h, "Nonbonded", self._interpolated)
        _apply_transforms(h, extra)
        return pot

    def set_exclusion_idxs(self, x):
        self.args[0] = x

    def get_exclusion_idxs(self):
        return self.args[0]

    def set_scale_factors(self, x):
        self.args[1] = x

    def get_scale_factors(self):
        return self.args[1]

    def get_lambda_plane_idxs(self):
        return self.args[2]

    def get_lambda_offset_idxs(self):
        return self.args[3]

    def set_lambda_plane_idxs(self, val):
        self.args[2] = val

    def set_lambda_offset_idxs(self, val):
        self.args[3] = val

    def get_beta(self):
        return self.args[4]

    def get_cutoff(self):
        return self.args[5]

    def interpolate(self):
        return NonbondedInterpolated(
            self.get_exclusion_idxs(),
            self.get_scale_factors(),
            self.get_lambda_plane_idxs(),
            self.get_lambda_offset_idxs(),
            self.get_beta(),
            self.get_cutoff(),
        )


class NonbondedInterpolated(Nonbonded):
    _interpolated = True


class _BondedWrapper(CustomOpWrapper):
    """timemachine/lib/potentials.py:162-196: args (idxs, lambda_mult=None, lambda_offset=None)."""

    _arity = 2
    _ctor = "tmnb_harmonic_bond_create"

    def unbound_impl(self, precision):
        if _check_precision(precision) != 32:
            raise RuntimeError(f"{type(self).__name__} is built with FP32 arithmetic only (precision=np.float32)")
        idxs = np.ascontiguousarray(self.args[0], dtype=np.int32).reshape(-1, self._arity)
        T = idxs.shape[0]
        mult = self.args[1] if len(self.args) > 1 else None
        off = self.args[2] if len(self.args) > 2 else None
        mult = None if mult is None else np.ascontiguousarray(mult, dtype=np.int32)
        off = None if off is None else np.ascontiguousarray(off, dtype=np.int32)
        h = ctypes.c_void_p()
        lib = _lib.lib()
        _lib.check(getattr(lib, self._ctor)(0, T, _ptr(idxs), _ptr(mult), _ptr(off), ctypes.byref(h)))
        return Potential(h, type(self).__name__, False)


class HarmonicBond(_BondedWrapper):
    _arity = 2
    _ctor = "tmnb_harmonic_bond_create"


class HarmonicAngle(_BondedWrapper):
    _arity = 3
    _ctor = "tmnb_harmonic_angle_create"


def all_flag_combinations():
    """The 16 (du_dx, du_dp, du_dl, u) request combinations (tests/common.py:451)."""
    return list(itertools.product([False, True], repeat=4))


__all__ += ["all_flag_combinations", "FIXED_EXPONENT", "HarmonicBond", "HarmonicAngle", "lambda_transform"]
