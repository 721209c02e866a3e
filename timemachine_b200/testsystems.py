"""Seeded synthetic water / ligand systems with timemachine's parameter conventions.

The reference's benchmark systems (DHFR in water, FreeSolv ligands) need
OpenMM and RDKit to parametrise; these builders produce systems of the same
shape and value distributions:

- rigid TIP3P-like waters: O on a cubic lattice with Gaussian jitter, H at
  0.09572 nm and 104.52 degrees in a uniformly random orientation;
- charges q * sqrt(138.935456) (O -0.834, H +0.417), LJ stored as sigma/2 and
  sqrt(epsilon) (O: sigma 0.315061 nm, eps 0.636386 kJ/mol; H: 0, 0)
  (timemachine/ff/handlers/openmm_deserializer.py:109,186-190);
- the three intramolecular pairs of each water excluded at full scale;
- a self-avoiding chain ligand with 0.15 nm bonds, charges N(0, 0.3) shifted to
  zero net charge, sigma ~ U(0.25, 0.38) nm, eps ~ U(0.1, 1.0) kJ/mol, 1-2 and
  1-3 pairs excluded, 1-4 pairs scaled by 0.5; ligand w offset = lambda * cutoff
  (lambda_offset_idxs = 1, lambda_plane_idxs = 0).
"""

from dataclasses import dataclass, field

import numpy as np

ONE_4PI_EPS0 = 138.935456
SQRT_K = np.sqrt(ONE_4PI_EPS0)
WATER_BOND = 0.09572
WATER_ANGLE = np.deg2rad(104.52)
O_SIGMA = 0.315061
O_EPS = 0.636386
MASS_O = 15.999
MASS_H = 1.008
MASS_LIG = 12.011
# flexible-water and ligand bonded constants (cosine-angle force constants)
WATER_KB = 345000.0
WATER_KA = 400.0
LIG_KB = 250000.0
LIG_B0 = 0.15
LIG_KA = 300.0
LIG_A0 = np.deg2rad(109.5)
# volume per water molecule at 1 g/cm^3 (nm^3): 18.015 g/mol / (602.214 nm^3 g/cm^3 per mol)
WATER_VOLUME = 18.015 / 602.214076


@dataclass
class System:
    x: np.ndarray  # (N, 3) float64, nm
    params: np.ndarray  # (N, 3) float64: q*sqrt(138.935456), sigma/2, sqrt(eps)
    box: np.ndarray  # (3, 3) float64
    exclusion_idxs: np.ndarray  # (E, 2) int32
    scales: np.ndarray  # (E, 2) float64 (charge, lj) fraction removed
    lambda_plane_idxs: np.ndarray  # (N,) int32
    lambda_offset_idxs: np.ndarray  # (N,) int32
    masses: np.ndarray  # (N,) float64 amu
    group_of: np.ndarray  # (N,) int32 molecule index (barostat groups)
    n_waters: int
    ligand_idxs: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.int32))
    beta: float = 2.0
    cutoff: float = 1.2
    # bonded terms (HarmonicBond [B,2] (kb, b0), HarmonicAngle [A,3] vertex-middle (ka, a0))
    bond_idxs: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), dtype=np.int32))
    bond_params: np.ndarray = field(default_factory=lambda: np.zeros((0, 2)))
    angle_idxs: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), dtype=np.int32))
    angle_params: np.ndarray = field(default_factory=lambda: np.zeros((0, 2)))

    @property
    def N(self):
        return self.x.shape[0]


def random_rotations(rng, n):
    """Uniform random rotation matrices (Shoemake's quaternion method)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    q = np.stack(
        [
            np.sqrt(1 - u1) * np.sin(2 * np.pi * u2),
            np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
            np.sqrt(u1) * np.sin(2 * np.pi * u3),
            np.sqrt(u1) * np.cos(2 * np.pi * u3),
        ],
        axis=1,
    )
    x, y, z, w = q.T
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def ligand_chain(rng, n_atoms, center, bond=0.15, min_sep=0.25, angle_deg=109.5):
    """Seeded self-avoiding chain: fixed bond length and angle, random torsions."""
    for _attempt in range(1000):
        pos = [np.zeros(3)]
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        pos.append(pos[0] + bond * d)
        ok = True
        theta = np.deg2rad(angle_deg)
        while len(pos) < n_atoms and ok:
            for _try in range(200):
                b1 = pos[-1] - pos[-2]
                b1 /= np.linalg.norm(b1)
                # random perpendicular direction
                r = rng.normal(size=3)
                r -= r.dot(b1) * b1
                r /= np.linalg.norm(r)
                new_dir = np.cos(np.pi - theta) * b1 + np.sin(np.pi - theta) * r
                cand = pos[-1] + bond * new_dir
                if len(pos) < 3 or np.min(np.linalg.norm(np.array(pos[:-2]) - cand, axis=1)) > min_sep:
                    pos.append(cand)
                    break
            else:
                ok = False
        if ok:
            p = np.array(pos)
            return p - p.mean(axis=0) + center
    raise RuntimeError("could not grow a self-avoiding ligand chain")


def ligand_topology(n_atoms):
    """Chain topology: 1-2 and 1-3 pairs excluded (scale 1), 1-4 pairs scaled by 0.5."""
    excl, scales = [], []
    for i in range(n_atoms):
        for k, s in ((1, 1.0), (2, 1.0), (3, 0.5)):
            j = i + k
            if j < n_atoms:
                excl.append((i, j))
                scales.append((s, s))
    return np.array(excl, dtype=np.int32).reshape(-1, 2), np.array(scales, dtype=np.float64).reshape(-1, 2)


def build_system(
    n_waters,
    box_edge,
    seed,
    n_ligand=0,
    jitter=0.02,
    hmr=False,
    cutoff=1.2,
    beta=2.0,
    ligand_offset=1,
):
    """Water box (lattice O + jitter) with an optional chain ligand at the centre."""
    rng = np.random.default_rng(seed)
    lig = None
    if n_ligand > 0:
        lig = ligand_chain(rng, n_ligand, center=np.full(3, box_edge / 2))
    n_side = int(np.ceil((n_waters + (n_ligand if n_ligand else 0)) ** (1.0 / 3.0) - 1e-9))
    while n_side**3 < n_waters:
        n_side += 1
    while True:
        spacing = box_edge / n_side
        g = (np.arange(n_side) + 0.5) * spacing
        lattice = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3)
        if lig is not None:
            # drop lattice sites nearest the ligand first, then random sites
            dmin = np.min(np.linalg.norm(lattice[:, None, :] - lig[None, :, :], axis=-1), axis=1)
            order = np.argsort(dmin)
            near = order[dmin[order] < 0.3]
            keep_mask = np.ones(len(lattice), dtype=bool)
            keep_mask[near] = False
            avail = np.flatnonzero(keep_mask)
        else:
            avail = np.arange(len(lattice))
        if len(avail) >= n_waters:
            break
        if spacing < 0.2:
            raise ValueError("box too small for the requested number of waters")
        n_side += 1  # the ligand displaced too many sites: a finer lattice
    chosen = np.sort(rng.choice(avail, size=n_waters, replace=False))
    O = lattice[chosen] + rng.normal(scale=jitter, size=(n_waters, 3))
    R = random_rotations(rng, n_waters)
    h = np.array(
        [
            [WATER_BOND * np.sin(WATER_ANGLE / 2), WATER_BOND * np.cos(WATER_ANGLE / 2), 0.0],
            [-WATER_BOND * np.sin(WATER_ANGLE / 2), WATER_BOND * np.cos(WATER_ANGLE / 2), 0.0],
        ]
    )
    H1 = O + np.einsum("nij,j->ni", R, h[0])
    H2 = O + np.einsum("nij,j->ni", R, h[1])
    xw = np.stack([O, H1, H2], axis=1).reshape(-1, 3)

    pw = np.zeros((n_waters, 3, 3))
    pw[:, 0] = [-0.834 * SQRT_K, O_SIGMA / 2, np.sqrt(O_EPS)]
    pw[:, 1] = [0.417 * SQRT_K, 0.0, 0.0]
    pw[:, 2] = [0.417 * SQRT_K, 0.0, 0.0]
    pw = pw.reshape(-1, 3)

    base = 3 * np.arange(n_waters, dtype=np.int32)
    ew = np.stack(
        [np.stack([base, base + 1], 1), np.stack([base, base + 2], 1), np.stack([base + 1, base + 2], 1)], axis=1
    ).reshape(-1, 2)
    sw = np.ones((ew.shape[0], 2))

    mw = np.tile([MASS_O, MASS_H, MASS_H], n_waters).astype(np.float64)
    if hmr:
        # hydrogen mass repartitioning: H -> 3 amu, taken from the bonded O
        mw = np.tile([MASS_O - 2 * (3.0 - MASS_H), 3.0, 3.0], n_waters).astype(np.float64)
    gw = np.repeat(np.arange(n_waters, dtype=np.int32), 3)

    N_w = 3 * n_waters
    if lig is not None:
        q = rng.normal(scale=0.3, size=n_ligand)
        q -= q.mean()
        sig = rng.uniform(0.25, 0.38, size=n_ligand)
        eps = rng.uniform(0.1, 1.0, size=n_ligand)
        pl = np.stack([q * SQRT_K, sig / 2, np.sqrt(eps)], axis=1)
        el, sl = ligand_topology(n_ligand)
        x = np.concatenate([xw, lig])
        params = np.concatenate([pw, pl])
        excl = np.concatenate([ew, el + N_w]).astype(np.int32)
        scales = np.concatenate([sw, sl])
        masses = np.concatenate([mw, np.full(n_ligand, MASS_LIG)])
        group_of = np.concatenate([gw, np.full(n_ligand, n_waters, dtype=np.int32)])
        lig_idxs = np.arange(N_w, N_w + n_ligand, dtype=np.int32)
    else:
        x, params, excl, scales, masses, group_of = xw, pw, ew.astype(np.int32), sw, mw, gw
        lig_idxs = np.zeros(0, dtype=np.int32)
    # bonded terms: O-H bonds and the H-O-H angle of every water; chain bonds/angles of the ligand
    bw = np.concatenate([np.stack([base, base + 1], 1), np.stack([base, base + 2], 1)]).astype(np.int32)
    bpw = np.tile([WATER_KB, WATER_BOND], (bw.shape[0], 1))
    aw = np.stack([base + 1, base, base + 2], 1).astype(np.int32)
    apw = np.tile([WATER_KA, WATER_ANGLE], (aw.shape[0], 1))
    if lig is not None:
        li = np.arange(n_ligand, dtype=np.int32) + N_w
        bl = np.stack([li[:-1], li[1:]], 1)
        al = np.stack([li[:-2], li[1:-1], li[2:]], 1)
        bond_idxs = np.concatenate([bw, bl])
        bond_params = np.concatenate([bpw, np.tile([LIG_KB, LIG_B0], (bl.shape[0], 1))])
        angle_idxs = np.concatenate([aw, al])
        angle_params = np.concatenate([apw, np.tile([LIG_KA, LIG_A0], (al.shape[0], 1))])
    else:
        bond_idxs, bond_params, angle_idxs, angle_params = bw, bpw, aw, apw
    N = x.shape[0]
    plane = np.zeros(N, dtype=np.int32)
    offset = np.zeros(N, dtype=np.int32)
    offset[lig_idxs] = ligand_offset
    return System(
        x=np.ascontiguousarray(x, dtype=np.float64),
        params=np.ascontiguousarray(params, dtype=np.float64),
        box=np.eye(3) * box_edge,
        exclusion_idxs=np.ascontiguousarray(excl, dtype=np.int32),
        scales=np.ascontiguousarray(scales, dtype=np.float64),
        lambda_plane_idxs=plane,
        lambda_offset_idxs=offset,
        masses=masses,
        group_of=group_of.astype(np.int32),
        n_waters=n_waters,
        ligand_idxs=lig_idxs,
        beta=beta,
        cutoff=cutoff,
        bond_idxs=np.ascontiguousarray(bond_idxs, dtype=np.int32),
        bond_params=np.ascontiguousarray(bond_params, dtype=np.float64),
        angle_idxs=np.ascontiguousarray(angle_idxs, dtype=np.int32),
        angle_params=np.ascontiguousarray(angle_params, dtype=np.float64),
    )


def water_box_3k(seed=2024):
    """1,000 waters (3,000 atoms) in a 3.104 nm cubic box, lambda offsets 0."""
    return build_system(1000, 3.104, seed)


def water_ligand_23k(seed=2024, hmr=True):
    """7,600 waters + 40-atom ligand (22,840 atoms) in a 6.1 nm cubic box."""
    return build_system(7600, 6.1, seed, n_ligand=40, hmr=hmr)


def system_of_size(n_atoms, seed, n_ligand=None, min_edge=2.7, hmr=False):
    """Water + ligand system of about n_atoms at 1 g/cm^3; the edge is raised to
    min_edge for very small systems so the box stays valid for a 1.2 nm cutoff."""
    rng = np.random.default_rng(seed)
    if n_ligand is None:
        n_ligand = int(rng.integers(20, 61))
    n_waters = max(1, (n_atoms - n_ligand) // 3)
    edge = max(min_edge, (n_waters * WATER_VOLUME) ** (1.0 / 3.0))
    return build_system(n_waters, edge, seed + 1, n_ligand=n_ligand, hmr=hmr)
