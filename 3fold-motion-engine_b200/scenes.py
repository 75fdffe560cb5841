"""Seeded synthetic scenes (the reference uses no dataset for this path).

* stack / lattice -- the reference's own fixtures (scripts/colored_vs_jacobi.py:100-112): boxes
  (0.3, 0.3, 0.2) resting-pitch apart in z, 0.35 m apart in x and y, dropped onto the ground.
* unit_cube_stack -- 16 unit cubes with 1 mm seeded xy jitter on the ground (the plain
  relaxed-Jacobi workload: 1 m cubes of 1 kg, i.e. density 1).
* random_boxes -- N boxes with per-axis edges uniform in [lo, hi], dropped from seeded uniform
  positions in an X x Y x Z volume without initial overlap, per-body friction uniform in a range
  (the 10 000-box coloured Gauss-Seidel workload).
"""
from __future__ import annotations

import numpy as np

PITCH = 0.205


def stack(K):
    return [[0.0, 0.0, 0.101 + k * PITCH] for k in range(K)]


def lattice(n_target, layers=2):
    side = int(np.ceil(np.sqrt(n_target / layers)))
    out = []
    for lz in range(layers):
        for iy in range(side):
            for ix in range(side):
                out.append([ix * 0.35, iy * 0.35, 0.101 + lz * PITCH])
    return out[:n_target]


def unit_cube_stack(K=16, seed=0):
    rng = np.random.default_rng(seed)
    j = rng.uniform(-1e-3, 1e-3, size=(K, 2))
    return [[float(j[k, 0]), float(j[k, 1]), 0.501 + 1.001 * k] for k in range(K)]


def random_boxes(n=10000, edge=(0.2, 0.6), box=(20.0, 20.0, 10.0), mu=(0.3, 0.8), density=1000.0,
                 seed_size=1, seed_pos=2, seed_mu=3, max_tries=200):
    """Returns dict(dims (n,3), centers (n,3), mu (n,), density (n,)).  Centres: x, y uniform in
    [-X/2, X/2], z uniform in [h/2, Z] with h the box height, rejection-sampled against the
    axis-aligned boxes already placed (a uniform grid of cell 2*max edge makes it O(n))."""
    rs, rp, rm = (np.random.default_rng(s) for s in (seed_size, seed_pos, seed_mu))
    dims = rs.uniform(edge[0], edge[1], size=(n, 3))
    cell = 2.0 * edge[1]
    grid = {}
    centers = np.zeros((n, 3))
    for i in range(n):
        h = dims[i]
        for _ in range(max_tries):
            c = np.array([rp.uniform(-box[0] / 2, box[0] / 2), rp.uniform(-box[1] / 2, box[1] / 2),
                          rp.uniform(h[2] / 2, box[2])])
            key = tuple((c // cell).astype(int))
            ok = True
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        for j in grid.get((key[0] + dx, key[1] + dy, key[2] + dz), ()):
                            if np.all(np.abs(centers[j] - c) < (dims[j] + h) / 2):
                                ok = False
                                break
                        if not ok:
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                break
        else:
            raise RuntimeError("random_boxes: could not place a box without overlap; enlarge the volume")
        centers[i] = c
        grid.setdefault(key, []).append(i)
    return dict(dims=dims, centers=centers, mu=rm.uniform(mu[0], mu[1], size=n), density=np.full(n, density))


def jittered_boxes(n, edge=(0.2, 0.6), height=10.0, mu=(0.3, 0.8), density=1000.0, rng=None, pitch=None):
    """n random boxes in a footprint scaled to n (the 10 000-box, 20 x 20 x 10 m drop's body
    density: side 20 sqrt(n / 10^4) m, at least 2 m), without overlap: each box gets its own cell
    of a lattice of pitch > the largest edge, drawn uniformly without replacement, and a uniform
    jitter that keeps it inside the cell.  Vectorised, so hundreds of scenes build in seconds."""
    rng = rng if rng is not None else np.random.default_rng(0)
    pitch = pitch if pitch is not None else edge[1] * 1.0 + 0.02
    side = max(2.0, 20.0 * np.sqrt(n / 1e4))
    nx = max(1, int(side / pitch))
    nz = max(1, int(height / pitch))
    while nx * nx * nz < n:
        nx += 1
    dims = rng.uniform(edge[0], edge[1], size=(n, 3))
    cells = rng.choice(nx * nx * nz, size=n, replace=False)
    ix, iy, iz = cells // (nx * nz), (cells // nz) % nx, cells % nz
    centers = np.stack([(ix + 0.5) * pitch - nx * pitch / 2, (iy + 0.5) * pitch - nx * pitch / 2,
                        (iz + 0.5) * pitch], axis=1)
    centers += rng.uniform(-1.0, 1.0, size=(n, 3)) * (pitch - dims) / 2
    return dict(dims=dims, centers=centers, mu=rng.uniform(mu[0], mu[1], size=n), density=np.full(n, density))


def batched_scenes(n_scenes=512, nmin=8, nmax=2000, seed_n=5, seed_mass=6, seed_boxes=1, heavy_frac=0.1,
                   heavy_factor=100.0):
    """The batched workload: body counts log-uniform in [nmin, nmax] (round(exp(U[ln nmin,
    ln nmax]))), boxes sized and placed as the random-box drop scaled to each scene's footprint,
    and heavy_frac of each scene's bodies at heavy_factor x density (mass ratios 100:1)."""
    rn, rm, rb = (np.random.default_rng(s) for s in (seed_n, seed_mass, seed_boxes))
    counts = np.round(np.exp(rn.uniform(np.log(nmin), np.log(nmax), n_scenes))).astype(int)
    out = []
    for n in counts:
        sc = jittered_boxes(int(n), rng=rb)
        heavy = rm.random(int(n)) < heavy_frac
        sc["density"] = np.where(heavy, sc["density"] * heavy_factor, sc["density"])
        out.append(sc)
    return out


def box_lattice(n=100000, edge=0.25, extent=(50.0, 50.0, 10.0), jitter=0.05, mu=0.6, density=1000.0, seed=4):
    """The stress scene: n cubes of one edge on a seeded random subset of a lattice filling
    extent (pitch >= 1.05 x edge), each displaced by up to jitter x pitch per axis (uniform), the
    lowest layer resting just above the ground."""
    rng = np.random.default_rng(seed)
    vol = extent[0] * extent[1] * extent[2]
    pitch = max(edge * 1.05, (vol / n) ** (1.0 / 3.0))
    nx, ny, nz = (max(1, int(e / pitch)) for e in extent)
    while nx * ny * nz < n:
        pitch *= 0.99
        nx, ny, nz = (max(1, int(e / pitch)) for e in extent)
    cells = np.sort(rng.choice(nx * ny * nz, size=n, replace=False))
    ix, iy, iz = cells // (ny * nz), (cells // nz) % ny, cells % nz
    j = jitter * min(pitch - edge, pitch) / 2 if pitch > edge else 0.0
    centers = np.stack([(ix + 0.5) * pitch - nx * pitch / 2, (iy + 0.5) * pitch - ny * pitch / 2,
                        edge / 2 + 1e-3 + iz * pitch], axis=1) + rng.uniform(-1.0, 1.0, (n, 3)) * j
    centers[:, 2] = np.maximum(centers[:, 2], edge / 2 + 1e-3)
    return dict(dims=np.full((n, 3), edge), centers=centers, mu=np.full(n, mu), density=np.full(n, density))


def stance_batch(B=4096, nv=18, nc=4, mu=0.5, seed=8, slide=(0.3, 0.1)):
    """B seeded contact problems of a legged stance: a floating base (6 velocity coordinates)
    and nc legs of (nv - 6) / nc joints each, every leg touching the ground once.  Per problem
    an SPD mass matrix M = A A^T / nv + diag(U[0.5, 2]); per contact the rows (normal, t1, t2) of
    J act on the base (linear part along the frame, angular part through a random lever arm)
    and on that leg's joints (Gaussian), nothing else.  The free velocity slides the base
    tangentially by `slide` (plus noise) and presses it into the ground, so most contacts slip.
    Returns J (B, 3 nc, nv), Minv (B, nv, nv), v_free (B, nv), mu (B, nc) as float64 arrays."""
    rng = np.random.default_rng(seed)
    per_leg = (nv - 6) // nc
    A = rng.standard_normal((B, nv, nv))
    M = A @ A.transpose(0, 2, 1) / nv + np.einsum("bi,ij->bij", rng.uniform(0.5, 2.0, (B, nv)), np.eye(nv))
    Minv = np.linalg.inv(M)
    J = np.zeros((B, 3 * nc, nv))
    frame = np.eye(3)[[2, 0, 1]]  # rows n = z, t1 = x, t2 = y
    for c in range(nc):
        r = rng.uniform(-0.4, 0.4, (B, 3))
        r[:, 2] = -0.3
        for k in range(3):
            d = frame[k]
            J[:, 3 * c + k, 0:3] = d
            J[:, 3 * c + k, 3:6] = np.cross(r, d)  # angular part: (r x d) . w
            J[:, 3 * c + k, 6 + per_leg * c:6 + per_leg * (c + 1)] = rng.standard_normal((B, per_leg)) * 0.3
    v_free = rng.standard_normal((B, nv)) * 0.05
    v_free[:, 0] += slide[0]
    v_free[:, 1] += slide[1]
    v_free[:, 2] -= 0.2
    return J, Minv, v_free, np.full((B, nc), float(mu))


def ncp_lattice(n=10000, half=0.1, spacing=0.35, z0=0.0999, dz=0.1999, mass=1.0, dt=1.0 / 240.0, mu=0.5):
    """The reference's exact-cone NCP timing fixture, LatticeWorld (ncp/ncp_gpu.py:1556-1665), as
    the arrays of one BlockScene: a two-layer lattice of n cubes of half-edge `half` at rest
    (ceil(sqrt(n / 2))^2 lower bodies on the ground, the rest stacked on the first of them), one
    ground pair per lower body and one stacking pair per upper body, each expanded to its four
    bottom corners (n_c = 4 n).  Normals are +z, the interface plane of a stacked pair passes
    through the lower centre + half, Ja/Jb are the rows (n, t1, t2) = (z, x, y) on (v, w), the
    free velocity is gravity's, and the bias is gap/dt when open, else the Baumgarte term.
    Returns a dict of BlockScene's fields (float64)."""
    g = int(np.ceil(np.sqrt(n / 2.0)))
    n_low = min(g * g, n)
    n_up = n - n_low
    ix, iy = np.divmod(np.arange(n_low), g)
    x = np.zeros((n, 3))
    x[:n_low, 0] = (ix - (g - 1) / 2.0) * spacing
    x[:n_low, 1] = (iy - (g - 1) / 2.0) * spacing
    x[:n_low, 2] = z0
    x[n_low:, :2] = x[:n_up, :2]
    x[n_low:, 2] = z0 + dz
    h = float(half)
    Ib = mass / 12.0 * ((2 * h) ** 2 + (2 * h) ** 2)
    off = np.array([[-h, -h, -h], [h, -h, -h], [-h, h, -h], [h, h, -h]])
    K = len(off)
    ca = np.concatenate([np.repeat(np.arange(n_low), K), np.repeat(np.arange(n_low, n), K)])
    cb = np.concatenate([np.full(n_low * K, -1), np.repeat(np.arange(n_up), K)])
    offs = np.tile(off, (n_low + n_up, 1))
    feat = (np.arange(len(ca)) % K).astype(np.int32) + 8 * (cb + 1).astype(np.int32)
    pa = x[ca] + offs  # identity orientations
    gap = np.empty(len(ca))
    gnd = cb < 0
    gap[gnd] = pa[gnd, 2]
    gap[~gnd] = pa[~gnd, 2] - (x[cb[~gnd], 2] + h)
    Minv = np.zeros((n, 6, 6))
    Minv[:, 0, 0] = Minv[:, 1, 1] = Minv[:, 2, 2] = 1.0 / mass
    Minv[:, 3, 3] = Minv[:, 4, 4] = Minv[:, 5, 5] = 1.0 / Ib
    vf = np.zeros((n, 6))
    vf[:, 2] = dt * (-9.81)
    D = np.array([[0.0, 0.0, 1.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]])
    nc = len(ca)
    ra = pa - x[ca]
    Ja = np.zeros((nc, 3, 6))
    Jb = np.zeros((nc, 3, 6))
    Ja[:, :, :3] = D
    Ja[:, :, 3:] = np.cross(ra[:, None, :], D[None, :, :])
    hasb = cb >= 0
    rb = np.zeros((nc, 3))
    rb[hasb] = pa[hasb] - x[cb[hasb]]
    Jb[hasb, :, :3] = -D
    Jb[hasb, :, 3:] = -np.cross(rb[hasb][:, None, :], D[None, :, :])
    bias = np.zeros((nc, 3))
    bias[:, 0] = np.where(gap > 0, gap / dt, -0.2 * np.maximum(-gap - 1e-4, 0.0) / dt)
    return dict(Ja=Ja, Jb=Jb, Minv=Minv, v_free=vf, mu=np.full(nc, float(mu)),
                body_pairs=np.stack([ca, cb], axis=1).astype(np.int32), dt=dt, bias=bias, feature=feat)


def pushed_pyramids(n_scenes=256, edge=0.2, density=1000.0, mu=0.5, plate_speed=0.2, seed_jitter=7, seed_target=8,
                    seed_v0=9, jitter=1e-3, target_sigma=0.05, v0_sigma=0.1):
    """The differentiable workload: `n_scenes` copies of a 64-box stepped pyramid pushed along +x
    by a kinematic plate.  A pyramid is four slices (along y, 3 mm apart) of layers 8-4-2-1-1
    boxes wide (x, 1 mm apart), each layer centred on the one below; edge 0.2 m, density 1000.
    Per scene: seeded uniform jitter of +-1 mm on every box position (seed 7), targets = the
    nominal positions + N(0, 0.05) m (seed 8), initial velocities N(0, 0.1) m/s (seed 9).  The plate
    (half extents 0.02 x 0.45 x 0.3, kinematic) starts 2 cm left of the base and moves at 0.2 m/s.
    Returns dict(half (n,3), mass (n,), x (n,3), kin (n,), v_kin (n,6), scene (n,), mu (n,),
    target (n,3), v0 (n,3)) over all scenes, the plate last in each scene (zero target and v0)."""
    rj, rt, rv = (np.random.default_rng(s) for s in (seed_jitter, seed_target, seed_v0))
    h = edge / 2
    pos = []
    widths = (8, 4, 2, 1, 1)
    for sl in range(4):
        y = (sl - 1.5) * (edge + 3e-3)
        for k, wdt in enumerate(widths):
            z = h + k * (edge + 1e-3)
            for i in range(wdt):
                pos.append([(i - (wdt - 1) / 2) * (edge + 1e-3), y, z])
    pos = np.array(pos)
    nb = len(pos)  # 64
    plate_half = np.array([0.02, 0.45, 0.3])
    plate_x = np.array([-(4 * (edge + 1e-3)) - 0.02 - plate_half[0], 0.0, plate_half[2] + 0.005])
    out = {k: [] for k in ("half", "mass", "x", "kin", "v_kin", "scene", "mu", "target", "v0")}
    for s in range(n_scenes):
        x = pos + rj.uniform(-jitter, jitter, size=pos.shape)
        out["x"].append(np.vstack([x, plate_x]))
        out["half"].append(np.vstack([np.full((nb, 3), h), plate_half]))
        out["mass"].append(np.r_[np.full(nb, density * edge ** 3), 1.0])
        out["kin"].append(np.r_[np.zeros(nb, np.int32), 1])
        vk = np.zeros((nb + 1, 6))
        vk[nb, 0] = plate_speed
        out["v_kin"].append(vk)
        out["scene"].append(np.full(nb + 1, s, np.int32))
        out["mu"].append(np.full(nb + 1, mu))
        out["target"].append(np.vstack([pos + rt.normal(0.0, target_sigma, size=pos.shape), np.zeros(3)]))
        out["v0"].append(np.vstack([rv.normal(0.0, v0_sigma, size=pos.shape), np.zeros(3)]))
    return {k: np.concatenate(v) for k, v in out.items()}
