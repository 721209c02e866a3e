"""Shared helpers of the test-suite (systems with the reference tests' shapes)."""

import numpy as np

from timemachine_b200 import testsystems

ONE_4PI_EPS0 = 138.935456


def random_params(rng, N, sigma_scale=5.0):
    """Random (q, sigma/2, sqrt(eps)) of the reference tests' magnitudes
    (tests/common.py:166-196)."""
    p = np.stack(
        [
            (rng.random(N) - 0.5) * np.sqrt(ONE_4PI_EPS0),
            rng.random(N) / sigma_scale,
            rng.random(N),
        ],
        axis=1,
    )
    p[:, 1] = p[:, 1] / 2
    p[:, 2] = np.sqrt(p[:, 2])
    return p


def water_exclusions(rng, N):
    """Water-style exclusions with random 1-3 scales (tests/common.py:199-224)."""
    excl, scales = [], []
    for i in range(N // 3):
        o, h1, h2 = 3 * i, 3 * i + 1, 3 * i + 2
        excl += [[o, h1], [o, h2], [h1, h2]]
        scales += [[1.0, 1.0], [1.0, 1.0], [rng.random(), rng.random()]]
    return np.array(excl, dtype=np.int32).reshape(-1, 2), np.array(scales, dtype=np.float64).reshape(-1, 2)


def small_water_case(rng, n_atoms, box_edge=3.0, p_scale=5.0, planes=(-2, 2), offsets=(-2, 2)):
    """Prefix of a synthetic 3 nm water box with random parameters and random
    4D plane/offset indices (tests/test_nonbonded.py:444-491 pattern)."""
    n_w = int(round(box_edge**3 / testsystems.WATER_VOLUME))
    s = testsystems.build_system(n_w, box_edge, seed=int(rng.integers(1 << 30)))
    x = s.x[:n_atoms]
    N = x.shape[0]
    params = random_params(rng, N, p_scale)
    excl, scales = water_exclusions(rng, N)
    plane = rng.integers(planes[0], planes[1], size=N, dtype=np.int32)
    offset = rng.integers(offsets[0], offsets[1], size=N, dtype=np.int32)
    return dict(x=x, params=params, box=s.box.copy(), exclusion_idxs=excl, scales=scales, plane=plane, offset=offset)


def f32_round(a):
    """Inputs as the reference tests feed them: rounded through float32 (tests/common.py:437-438)."""
    return np.asarray(a, dtype=np.float32).astype(np.float64)
