"""Seeded synthetic inputs for the benchmark and parity workloads.

No public dataset is involved: molecules are random atoms of a protein-like
composition (C 62 %, N 17 %, O 20 %, S 1 %, exact rounded counts, shuffled)
placed uniformly in a ball with a 1.2 Angstrom minimum separation, and
rotations are Haar-uniform (Shoemake's quaternion construction).  Seeds are
NumPy PCG64 streams, 1000 + workload index unless given.
"""
import numpy as np

COMPOSITION = ((6, 0.62), (7, 0.17), (8, 0.20), (16, 0.01))
MIN_SEPARATION = 1.2e-10  # m


def composition_counts(n):
    """Exact rounded element counts summing to n (largest remainders)."""
    raw = np.array([f * n for _, f in COMPOSITION])
    cnt = np.floor(raw).astype(int)
    rest = n - cnt.sum()
    order = np.argsort(-(raw - cnt))
    for k in range(rest):
        cnt[order[k % len(cnt)]] += 1
    return {z: int(c) for (z, _), c in zip(COMPOSITION, cnt)}


def random_molecule(n, radius, seed, min_sep=MIN_SEPARATION):
    """(Z int32[n], pos float32[n,3] metres) uniform in a ball of `radius` metres."""
    from scipy.spatial import cKDTree

    rng = np.random.Generator(np.random.PCG64(seed))
    counts = composition_counts(n)
    Z = np.concatenate([np.full(c, z, np.int32) for z, c in counts.items()])
    rng.shuffle(Z)
    pts = np.empty((0, 3))
    while pts.shape[0] < n:
        m = int((n - pts.shape[0]) * 1.4) + 64
        d = rng.normal(size=(m, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        r = radius * rng.random(m) ** (1.0 / 3.0)
        cand = np.concatenate([pts, d * r[:, None]])
        tree = cKDTree(cand)
        drop = set()
        for i, j in sorted(tree.query_pairs(min_sep)):
            if i not in drop and j not in drop:
                drop.add(max(i, j))
        keep = np.array([k for k in range(cand.shape[0]) if k not in drop], dtype=int)
        pts = cand[keep][:n]
    return Z, pts.astype(np.float32)


def haar_rotations(n, seed):
    """n Haar-uniform 3x3 rotation matrices (float64), Shoemake (1992)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a, b = np.sqrt(1 - u1), np.sqrt(u1)
    w, x = a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2)
    y, z = b * np.sin(2 * np.pi * u3), b * np.cos(2 * np.pi * u3)
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


def detector(nx, pixel, distance, wavelength):
    """Square flat detector centred on the beam, as keyword arguments."""
    return dict(nx=nx, ny=nx, width=nx * pixel, height=nx * pixel, distance=distance, wavelength=wavelength)


# The five workloads (atoms, ball radius, detector) as described for the benchmark.
WORKLOADS = {
    "plain_1k": dict(natoms=1000, radius=2.5e-9, det=detector(256, 75e-6, 0.15, 0.25e-9), seed=1000),
    "precision_50k": dict(natoms=50000, radius=12e-9, det=detector(1024, 75e-6, 0.1, 0.15e-9), seed=1001,
                          readout_noise=10.0, full_well_clamp=65535.0),
    "orientations_20k": dict(natoms=20000, radius=8e-9, det=detector(256, 150e-6, 0.2, 0.2e-9), seed=1002,
                             n_orient=4096, rot_seed=3003),
    "uneven_64": dict(n_mol=64, seed=1003, density=50e27),
    "adjoint_5k": dict(natoms=5000, radius=4e-9, det=detector(512, 75e-6, 0.15, 0.25e-9), seed=1004,
                       n_orient=256, rot_seed=3004),
}


def uneven_batch(seed=1003, n_mol=64, density=50e27, sizes=(128, 256, 512, 1024), nmin=500, nmax=100000):
    """Molecules with atom counts log-uniform in [nmin, nmax], radius from `density`
    (atoms / m^3, protein-like 50 / nm^3), each with its own detector drawn from
    `sizes` at 0.15 m / 75 um and a wavelength uniform in [0.1, 0.3] nm."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(n_mol):
        n = int(round(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))
        radius = (3 * n / (4 * np.pi * density)) ** (1.0 / 3.0)
        nx = int(rng.choice(sizes))
        lam = float(rng.uniform(0.1e-9, 0.3e-9))
        out.append(dict(natoms=n, radius=radius, det=detector(nx, 75e-6, 0.15, lam), seed=seed * 1000 + i))
    return out
