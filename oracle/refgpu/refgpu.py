"""ctypes wrapper of the reference timemachine CUDA build (TEST INFRASTRUCTURE; also timed by the reference arm of bench.py).

Loads oracle/_ref/libtmref.so (built from the reference sources by
oracle/refgpu/Makefile) for the bit-exact parity tests and for bench.py's
reference arm. The product never imports this module.
"""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(os.path.dirname(HERE), "_ref")
LIB_PATH = os.path.join(REF_DIR, "libtmref.so")
KERNEL_DIR = os.path.join(REF_DIR, "kernels")

_lib = None


def available():
    return os.path.exists(LIB_PATH) and os.path.exists(os.path.join(KERNEL_DIR, "k_lambda_transformer_jit.cuh"))


def build(reference_root=None):
    """Build oracle/_ref from the reference tree (only where the tree exists):
    reference_root, else $TMNB_REFERENCE_ROOT."""
    import subprocess

    reference_root = reference_root or os.environ.get("TMNB_REFERENCE_ROOT")
    if not reference_root or not os.path.isdir(reference_root):
        return False
    subprocess.run(["make", "-C", HERE, f"REF={reference_root}", "-j8"], check=True)
    return True


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise ImportError(f"{LIB_PATH} not built (make -C oracle/refgpu)")
        L = ctypes.CDLL(LIB_PATH)
        vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.tmref_last_error.restype = ctypes.c_char_p
        L.tmref_nonbonded_create.restype = vp
        cp = ctypes.c_char_p
        L.tmref_nonbonded_create.argtypes = [cp, i, vp, vp, i, vp, vp, d, d, i, i, cp, cp, cp, cp]
        L.tmref_nonbonded_destroy.argtypes = [vp]
        L.tmref_set_nblist_padding.argtypes = [vp, d]
        L.tmref_disable_hilbert_sort.argtypes = [vp]
        L.tmref_execute_device.argtypes = [vp, i, i, vp, vp, vp, d, vp, vp, vp, vp, vp]
        L.tmref_execute_host.argtypes = [vp, i, i, vp, vp, vp, d, vp, vp, vp, vp]
        L.tmref_group_create.restype = vp
        L.tmref_group_create.argtypes = [ctypes.c_char_p, i, vp, i, vp, vp, d, d, i, i]
        L.tmref_pot_destroy.argtypes = [vp]
        L.tmref_pot_execute_host.argtypes = [vp, i, i, vp, vp, vp, d, vp, vp, vp, vp]
        L.tmref_md_create.restype = vp
        L.tmref_md_create.argtypes = [vp, i, vp, i, vp, vp, vp, d, d, vp, vp, i, d, d, vp, i, vp, i, vp, vp, i, vp]
        L.tmref_md_run.argtypes = [vp, i, d, vp, vp]
        L.tmref_md_destroy.argtypes = [vp]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().tmref_last_error().decode())


class RefNonbonded:
    """FanoutSummedPotential([NonbondedAllPairs_f32, NonbondedPairList_f32_negated]) of the reference
    (the _f64 kernels with precision=64; transforms: the four lambda-transform expressions)."""

    def __init__(self, exclusion_idxs, scales, plane, offset, beta, cutoff, interpolated=False, precision=32,
                 transforms=None):
        L = lib()
        exclusion_idxs = np.asarray(exclusion_idxs).reshape(-1, 2)
        scales = np.asarray(scales).reshape(-1, 2)
        if exclusion_idxs.shape[0] == 0:
            # the reference's pair-list launch has an empty grid for zero pairs
            # (invalid configuration -> exit); a zero-scale pair contributes 0
            exclusion_idxs = np.array([[0, 1]])
            scales = np.zeros((1, 2))
        self._keep = [
            np.ascontiguousarray(exclusion_idxs, dtype=np.int32).reshape(-1, 2),
            np.ascontiguousarray(scales, dtype=np.float64).reshape(-1, 2),
            np.ascontiguousarray(plane, dtype=np.int32),
            np.ascontiguousarray(offset, dtype=np.int32),
        ]
        e, s, pl, of = self._keep
        self.N = pl.size
        self.interpolated = interpolated
        t = [None] * 4 if transforms is None else [x.encode() for x in transforms]
        self._h = L.tmref_nonbonded_create(
            KERNEL_DIR.encode(), pl.size, _p(e), _p(s), e.shape[0], _p(pl), _p(of), beta, cutoff,
            1 if interpolated else 0, int(precision), *t,
        )
        if not self._h:
            raise RuntimeError(L.tmref_last_error().decode())

    def __del__(self):
        if getattr(self, "_h", None):
            lib().tmref_nonbonded_destroy(self._h)
            self._h = None

    def set_nblist_padding(self, p):
        _check(lib().tmref_set_nblist_padding(self._h, float(p)))

    def disable_hilbert_sort(self):
        _check(lib().tmref_disable_hilbert_sort(self._h))

    def execute_device(self, x, p, box, lam, du_dx=None, du_dp=None, du_dl=None, u=None, stream=0):
        def a(t):
            return None if t is None else ctypes.c_void_p(t.data_ptr())

        _check(
            lib().tmref_execute_device(
                self._h, x.shape[0], p.numel(), a(x), a(p), a(box), float(lam), a(du_dx), a(du_dp), a(du_dl), a(u),
                ctypes.c_void_p(stream),
            )
        )

    def execute_host_fixed(self, x, p, box, lam, du_dx=True, du_dp=True, du_dl=True, u=True):
        x = np.ascontiguousarray(x, dtype=np.float64)
        p = np.ascontiguousarray(p, dtype=np.float64)
        box = np.ascontiguousarray(box, dtype=np.float64)
        N = x.shape[0]
        o = [
            np.zeros((N, 3), np.uint64) if du_dx else None,
            np.zeros(p.size, np.uint64) if du_dp else None,
            np.zeros(N, np.uint64) if du_dl else None,
            np.zeros(N, np.uint64) if u else None,
        ]
        _check(lib().tmref_execute_host(self._h, N, p.size, _p(x), _p(p), _p(box), float(lam), *[_p(t) for t in o]))
        return o


class RefInteractionGroup:
    """NonbondedInteractionGroup(_Interpolated)_f32 (or _f64, precision=64) of the reference."""

    def __init__(self, row_idxs, plane, offset, beta, cutoff, interpolated=False, precision=32):
        L = lib()
        self._keep = [
            np.ascontiguousarray(row_idxs, dtype=np.int32),
            np.ascontiguousarray(plane, dtype=np.int32),
            np.ascontiguousarray(offset, dtype=np.int32),
        ]
        r, pl, of = self._keep
        self._h = L.tmref_group_create(
            KERNEL_DIR.encode(), pl.size, _p(r), r.size, _p(pl), _p(of), beta, cutoff, 1 if interpolated else 0,
            int(precision),
        )
        if not self._h:
            raise RuntimeError(L.tmref_last_error().decode())

    def __del__(self):
        if getattr(self, "_h", None):
            lib().tmref_pot_destroy(self._h)
            self._h = None

    def execute_host_fixed(self, x, p, box, lam):
        x = np.ascontiguousarray(x, dtype=np.float64)
        p = np.ascontiguousarray(p, dtype=np.float64)
        box = np.ascontiguousarray(box, dtype=np.float64)
        N = x.shape[0]
        o = [np.zeros((N, 3), np.uint64), np.zeros(p.size, np.uint64), np.zeros(N, np.uint64), np.zeros(N, np.uint64)]
        _check(lib().tmref_pot_execute_host(self._h, N, p.size, _p(x), _p(p), _p(box), float(lam), *[_p(t) for t in o]))
        return o


class RefMD:
    """Reference Context(LangevinIntegrator, [Nonbonded], MonteCarloBarostat)."""

    def __init__(
        self, nb, params, x0, v0, box, dt, ca, cbs, ccs, seed, pressure, temperature, group_of, interval,
        bond_idxs=None, bond_params=None, angle_idxs=None, angle_params=None,
    ):
        L = lib()
        self._keep = [
            np.ascontiguousarray(params, dtype=np.float64),
            np.ascontiguousarray(x0, dtype=np.float64),
            np.ascontiguousarray(v0, dtype=np.float64),
            np.ascontiguousarray(box, dtype=np.float64),
            np.ascontiguousarray(cbs, dtype=np.float64),
            np.ascontiguousarray(ccs, dtype=np.float64),
            np.ascontiguousarray(group_of, dtype=np.int32),
        ]
        pp, xx, vv, bb, cb, cc, gg = self._keep
        bi = np.ascontiguousarray(np.zeros((0, 2)) if bond_idxs is None else bond_idxs, dtype=np.int32)
        bpar = np.ascontiguousarray(np.zeros((0, 2)) if bond_params is None else bond_params, dtype=np.float64)
        ai = np.ascontiguousarray(np.zeros((0, 3)) if angle_idxs is None else angle_idxs, dtype=np.int32)
        apar = np.ascontiguousarray(np.zeros((0, 2)) if angle_params is None else angle_params, dtype=np.float64)
        self._keep += [bi, bpar, ai, apar]
        self.nb = nb
        self.N = xx.shape[0]
        self._h = L.tmref_md_create(
            nb._h, self.N, _p(pp), pp.size, _p(xx), _p(vv), _p(bb), dt, ca, _p(cb), _p(cc), seed, pressure,
            temperature, _p(gg), interval, _p(bi), bi.shape[0], _p(bpar), _p(ai), ai.shape[0], _p(apar),
        )
        if not self._h:
            raise RuntimeError(L.tmref_last_error().decode())

    def run(self, n_steps, lam=0.0):
        x = np.zeros((self.N, 3))
        box = np.zeros((3, 3))
        _check(lib().tmref_md_run(self._h, n_steps, float(lam), _p(x), _p(box)))
        return x, box

    def __del__(self):
        if getattr(self, "_h", None):
            lib().tmref_md_destroy(self._h)
            self._h = None
