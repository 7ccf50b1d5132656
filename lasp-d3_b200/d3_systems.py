"""Seeded synthetic structures for the D3 workloads.

Every generator is deterministic in its seed and returns a dict with
  pos   float64 [n, 3]  Cartesian positions, Angstrom
  Z     int array [n]   atomic numbers
  cell  float64 [3, 3]  rows are lattice vectors, Angstrom

Workloads (no public dataset is involved; these stand in with the stated shapes):
  water_box      32 rigid H2O in a 9.86 A cubic cell (96 atoms)
  random_box     uniform positions with a 1.0 A minimum-image rejection, given cell
                 rows and composition (the 20,000-atom triclinic box and its scaled
                 250,000 / 100,000-atom variants)
  batch_structs  many small sheared cubic cells at 0.1 atoms/A^3 with Dirichlet(1)
                 compositions (the 2,048-structure batch)
  gtest_*        the property-test systems of the reference's test/d3_test.cpp:343-417
"""
import numpy as np

Z_OF = {"H": 1, "C": 6, "N": 7, "O": 8, "Si": 14, "Fe": 26, "Cu": 29}

TRICLINIC_58 = np.array([[58.0, 0.0, 0.0], [5.0, 58.0, 0.0], [3.0, 4.0, 58.0]])
MIX_HCNOCU = (("H", 0.40), ("C", 0.30), ("N", 0.10), ("O", 0.15), ("Cu", 0.05))


def _min_image_frac(df):
    return df - np.round(df)


def _random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def water_box(seed=0, edge=9.86, grid=(4, 4, 2), jitter=0.3, min_oo=2.5, r_oh=0.9572, angle_deg=104.52):
    """32 rigid waters: O on a jittered grid (min-image O-O >= min_oo), random orientations."""
    rng = np.random.default_rng(seed)
    cell = np.eye(3) * edge
    base = np.array([((i + 0.5) / grid[0], (j + 0.5) / grid[1], (k + 0.5) / grid[2])
                     for i in range(grid[0]) for j in range(grid[1]) for k in range(grid[2])]) * edge
    m = len(base)
    jit = rng.uniform(-jitter, jitter, (m, 3))

    def violations(p):
        d = p[:, None, :] - p[None, :, :]
        d -= np.round(d / edge) * edge
        r = np.linalg.norm(d, axis=2) + np.eye(m) * 1e9
        return r < min_oo

    # rejection with local repair: re-draw the jitter of one offending molecule at a
    # time, keeping a re-draw only when it does not add violations
    for _it in range(200000):
        bad = violations(base + jit)
        nbad = int(bad.sum())
        if nbad == 0:
            break
        i = int(rng.choice(np.nonzero(bad.any(axis=1))[0]))
        old = jit[i].copy()
        jit[i] = rng.uniform(-jitter, jitter, 3)
        if int(violations(base + jit).sum()) > nbad:
            jit[i] = old
    else:
        raise RuntimeError("water_box: rejection sampling failed")
    ox = base + jit
    half = np.deg2rad(angle_deg) / 2
    h1 = r_oh * np.array([np.sin(half), np.cos(half), 0.0])
    h2 = r_oh * np.array([-np.sin(half), np.cos(half), 0.0])
    pos, Z = [], []
    for o in ox:
        R = _random_rotation(rng)
        pos += [o, o + R @ h1, o + R @ h2]
        Z += [8, 1, 1]
    return {"pos": np.array(pos), "Z": np.array(Z), "cell": cell}


def _cell_heights(cell):
    inv = np.linalg.inv(cell)
    return 1.0 / np.linalg.norm(inv, axis=0)


def random_box(n, cell, composition=MIX_HCNOCU, seed=1, rmin=1.0, chunk=None):
    """Uniform random positions in a (triclinic) periodic cell with min-image rejection
    at rmin, and an exact-count random composition."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    cell = np.asarray(cell, float)
    h = _cell_heights(cell)
    margin = rmin / h + 1e-9
    shifts = np.array([(i, j, k) for i in (-1, 0, 1) for j in (-1, 0, 1) for k in (-1, 0, 1)], float)
    acc = np.zeros((0, 3))
    while len(acc) < n:
        m = max(64, int((n - len(acc)) * 1.15))
        cand = rng.uniform(0.0, 1.0, size=(m, 3))
        # images of accepted atoms near the faces
        if len(acc):
            imgs = []
            for s in shifts:
                f = acc + s
                keep = np.all((f > -margin) & (f < 1 + margin), axis=1)
                imgs.append(f[keep])
            tree = cKDTree(np.concatenate(imgs) @ cell)
            d, _ = tree.query(cand @ cell, k=1, distance_upper_bound=rmin)
            cand = cand[~np.isfinite(d)]
        # conflicts inside the chunk: keep the earlier candidate
        imgs, owner = [], []
        for s in shifts:
            f = cand + s
            keep = np.nonzero(np.all((f > -margin) & (f < 1 + margin), axis=1))[0]
            imgs.append(f[keep])
            owner.append(keep)
        owner = np.concatenate(owner)
        tree = cKDTree(np.concatenate(imgs) @ cell)
        pairs = tree.query_pairs(rmin, output_type="ndarray")
        drop = np.zeros(len(cand), bool)
        if len(pairs):
            a, b = owner[pairs[:, 0]], owner[pairs[:, 1]]
            sel = a != b
            a, b = a[sel], b[sel]
            lo, hi = np.minimum(a, b), np.maximum(a, b)
            order = np.lexsort((hi, lo))
            for x, y in zip(lo[order], hi[order]):
                if not drop[x]:
                    drop[y] = True
        cand = cand[~drop]
        acc = np.concatenate([acc, cand[: n - len(acc)]])
    pos = acc @ cell
    # largest-remainder apportionment of n atoms over the composition fractions
    frac = np.array([f for _, f in composition], float)
    frac = frac / frac.sum()
    raw = frac * n
    counts = np.floor(raw).astype(int)
    for k in np.argsort(-(raw - counts))[: n - counts.sum()]:
        counts[k] += 1
    counts = counts.tolist()
    Z = np.concatenate([np.full(c, Z_OF[s]) for (s, _), c in zip(composition, counts)])
    rng.shuffle(Z)
    return {"pos": pos, "Z": Z, "cell": cell}


def triclinic_box(n=20000, seed=1, composition=MIX_HCNOCU):
    """The 20,000-atom triclinic box (a=(58,0,0), b=(5,58,0), c=(3,4,58) A); for other n
    the cell edges are scaled by (n/20000)^(1/3) keeping the tilt ratios."""
    cell = TRICLINIC_58 * (n / 20000.0) ** (1.0 / 3.0)
    return random_box(n, cell, composition=composition, seed=seed)


def cell_list_box(n=400, seed=31, edge=160.0, shear=0.0):
    """A low-density box thick enough (every perpendicular height above 3 x 95 bohr) for
    the reference's cell-list path. shear: the b vector's x component in units of the
    edge, which makes the reference's grid cells along x thinner than the cutoff."""
    cell = edge * np.array([[1.0, 0.0, 0.0], [shear, 1.0, 0.0], [0.0, 0.0, 1.0]])
    return random_box(n, cell, composition=MIX_HCNOCU, seed=seed)


def batch_structs(count=2048, seed=3, nmin=8, nmax=2000, density=0.1, tilt=0.1,
                  species=("H", "C", "N", "O", "Si", "Cu")):
    """Independent periodic structures: log-uniform atom counts, cubic edge for the given
    density, sheared by uniform tilts, Dirichlet(1) composition per structure."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(count):
        n = int(round(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))
        L = (n / density) ** (1.0 / 3.0)
        t = rng.uniform(-tilt, tilt, 3)
        cell = L * np.array([[1.0, 0.0, 0.0], [t[0], 1.0, 0.0], [t[1], t[2], 1.0]])
        frac = rng.dirichlet(np.ones(len(species)))
        comp = tuple(zip(species, frac))
        out.append(random_box(n, cell, composition=comp, seed=int(rng.integers(1 << 31))))
    return out


# ---- reference property-test systems (test/d3_test.cpp:343-417) ----

def gtest_small_system():
    pos = np.array([[5.1372, 5.5512, 10.1047], [4.5169, 6.1365, 11.3604], [6.1937, 4.4752, 10.2703],
                    [4.7872, 5.9358, 8.9937], [6.7474, 4.3475, 9.3339], [5.6975, 3.5214, 10.5181],
                    [6.8870, 4.7006, 11.0939], [4.8579, 5.6442, 12.2774], [3.4204, 6.0677, 11.2935],
                    [4.7678, 7.2075, 11.4098]], np.float32).astype(np.float64)
    return {"pos": pos, "Z": np.array([6, 6, 6, 8, 1, 1, 1, 1, 1, 1]), "cell": np.eye(3) * 20.0}


def gtest_bcc_fe(surface=False):
    a = np.float32(2.87)
    pos = []
    for i in range(2):
        for j in range(2):
            for k in range(2):
                pos.append([i * a, j * a, k * a])
                pos.append([(i + np.float32(0.5)) * a, (j + np.float32(0.5)) * a, (k + np.float32(0.5)) * a])
    cell = np.diag([2 * a, 2 * a, 2 * a]).astype(np.float32)
    if surface:
        cell[2, 2] = cell[2, 2] * np.float32(1.2)
    return {"pos": np.array(pos, np.float32).astype(np.float64), "Z": np.full(16, 26),
            "cell": cell.astype(np.float64)}


def supercell(sys, reps=(2, 2, 2)):
    pos, Z = [], []
    for x in range(reps[0]):
        for y in range(reps[1]):
            for z in range(reps[2]):
                sh = x * sys["cell"][0] + y * sys["cell"][1] + z * sys["cell"][2]
                pos.append(sys["pos"] + sh)
                Z.append(sys["Z"])
    cell = sys["cell"] * np.array(reps)[:, None]
    return {"pos": np.concatenate(pos), "Z": np.concatenate(Z), "cell": cell}
