"""Regenerates the golden input fixtures from the reference's own test data.

Run in a container that has the reference tree (it is not needed afterwards):

    python tests/golden/make_golden.py [/path/to/timemachine]

The reference pickles hold timemachine objects; a stub unpickler maps every
timemachine class to a plain attribute bag, so no timemachine import (and no
jax) is needed. Each fixture is saved as a compressed .npz with the arrays the
tests need:

- bad_test_547.npz  (tests/data/bad_test_547.pkl.gz; tests/test_nonbonded.py:303-320):
  NonbondedInterpolated, 6316 atoms, lambda = 1.0; reference result du_dl == 0.
- repro.npz         (tests/data/repro.pkl.gz; tests/test_nonbonded.py:322-342):
  NonbondedInterpolated, 8873 atoms, lambda = 0; Hilbert on/off bitwise equality.
- water.npz         (tests/data/water.npy): 2997 water coordinates (nm).
"""

import gzip
import os
import pickle
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


class _Bag:
    def __init__(self, *a, **k):
        pass

    def __setstate__(self, state):
        if isinstance(state, dict):
            self.__dict__.update(state)
        else:
            self.__dict__["state"] = state


class _StubUnpickler(pickle.Unpickler):
    def find_class(self, module, name):
        if module.startswith("timemachine"):
            return type(name, (_Bag,), {})
        return super().find_class(module, name)


def load_pickle(path):
    with gzip.open(path, "rb") as f:
        return _StubUnpickler(f).load()


def convert(ref_root):
    data = os.path.join(ref_root, "tests", "data")
    for name in ["bad_test_547", "repro"]:
        x, box, lam, pot = load_pickle(os.path.join(data, name + ".pkl.gz"))
        args = pot.args
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"),
            kind=type(pot).__name__,
            x=np.asarray(x, dtype=np.float64),
            box=np.asarray(box, dtype=np.float64),
            lam=float(lam),
            exclusion_idxs=np.asarray(args[0], dtype=np.int32),
            scales=np.asarray(args[1], dtype=np.float64),
            lambda_plane_idxs=np.asarray(args[2], dtype=np.int32),
            lambda_offset_idxs=np.asarray(args[3], dtype=np.int32),
            beta=float(args[4]),
            cutoff=float(args[5]),
            params=np.asarray(pot.params, dtype=np.float64),
        )
    w = np.load(os.path.join(data, "water.npy"))
    np.savez_compressed(os.path.join(HERE, "water.npz"), x=np.asarray(w, dtype=np.float64))


if __name__ == "__main__":
    # the reference source tree: first argument, else $TMNB_REFERENCE_ROOT
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TMNB_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py <reference tree>  (or set TMNB_REFERENCE_ROOT)")
    convert(root)
