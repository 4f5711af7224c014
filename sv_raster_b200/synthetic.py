"""Seeded synthetic sparse-voxel scenes and cameras.

Stands in for the reference's datasets (none are available here): sparse
octree voxels inside the scene cube [-0.5, 0.5]^3 (scene centre 0, extent 1,
so a level-l voxel has edge 2^-l), with the reference's octree encoding:

* ``octpath``: 3 bits per level, level-1 octant in bits 45-47, deeper levels
  below, then zero-padded to 16 levels (``ijk_2_octpath``, utils.cu:129-158);
* voxel centre ``-0.5 + (ijk + 0.5) * 2^-l`` and size ``2^-l``
  (``octpath_decoding``, utils/octree_utils.py:99-126);
* no voxel overlaps another (no ancestor/descendant pairs), as in a valid
  SVRaster model.

Cameras are OpenCV pinholes (x right, y down, z forward) with row-major 4x4
``w2c`` and ``c2w = inverse(w2c)`` (cameras.py:119-155), principal point at the
image centre.  All randomness comes from ``numpy.random.default_rng(seed)``.
"""
import math
import os
import pickle
from dataclasses import dataclass, field

import numpy as np

MAX_LEVELS = 16


def ijk_to_octpath(ijk, level, max_levels=MAX_LEVELS):
    """(i,j,k) integer cell coords at `level` -> octpath (int64) of an octree
    `max_levels` deep (16, or 21 for the new_cuda encoding)."""
    ijk = np.asarray(ijk, dtype=np.int64)
    level = np.asarray(level, dtype=np.int64).reshape(-1)
    i, j, k = ijk[:, 0].copy(), ijk[:, 1].copy(), ijk[:, 2].copy()
    path = np.zeros(len(level), dtype=np.int64)
    for l in range(max_levels):
        bits = ((i & 1) << 2) | ((j & 1) << 1) | (k & 1)
        path |= bits << (3 * l)
        i >>= 1
        j >>= 1
        k >>= 1
    return path << (3 * (max_levels - level))


def octpath_to_ijk(path, level, max_levels=MAX_LEVELS):
    path = np.asarray(path, dtype=np.int64).reshape(-1)
    level = np.asarray(level, dtype=np.int64).reshape(-1)
    p = path >> (3 * (max_levels - level))
    ijk = np.zeros((len(path), 3), dtype=np.int64)
    for l in range(max_levels):
        bits = p & 7
        ijk[:, 0] |= ((bits >> 2) & 1) << l
        ijk[:, 1] |= ((bits >> 1) & 1) << l
        ijk[:, 2] |= (bits & 1) << l
        p >>= 3
    return ijk


def decode_voxels(path, level, max_levels=MAX_LEVELS):
    """Voxel centres [N,3] and sizes [N,1] (float32, exact) of octree cells."""
    ijk = octpath_to_ijk(path, level, max_levels)
    size = np.ldexp(1.0, -np.asarray(level, dtype=np.int64).reshape(-1, 1))
    centers = -0.5 + (ijk + 0.5) * size
    return centers.astype(np.float32), size.astype(np.float32)


def _cell_key(ijk, level):
    level = np.asarray(level, dtype=np.int64)
    side = np.left_shift(np.int64(1), level)
    return ((level << 52) | (ijk[:, 0] * side * side + ijk[:, 1] * side + ijk[:, 2])).astype(np.int64)


def _cells_from_points(pts, levels):
    side = np.left_shift(np.int64(1), levels.astype(np.int64))
    ijk = np.floor((pts + 0.5) * side[:, None]).astype(np.int64)
    ijk = np.clip(ijk, 0, side[:, None] - 1)
    return ijk


def remove_overlaps(ijk, level):
    """Unique non-overlapping cells: a cell is dropped when any ancestor is present.

    Returns the indices (into the inputs) of kept cells, in input order of first
    occurrence.
    """
    level = np.asarray(level, dtype=np.int64)
    keys = _cell_key(ijk, level)
    _, first = np.unique(keys, return_index=True)
    first = np.sort(first)
    ijk, level = ijk[first], level[first]
    keys = keys[first]
    keep = np.ones(len(first), dtype=bool)
    present_levels = np.unique(level)
    sorted_keys = np.sort(keys)
    for l in present_levels:
        sel = np.where(level == l)[0]
        for la in present_levels:
            if la >= l:
                break
            anc = ijk[sel] >> (l - la)
            akeys = _cell_key(anc, np.full(len(sel), la))
            pos = np.searchsorted(sorted_keys, akeys)
            pos = np.minimum(pos, len(sorted_keys) - 1)
            hit = sorted_keys[pos] == akeys
            keep[sel[hit]] = False
    return first[keep]


def _sphere_points(rng, n, center, radius, jitter):
    d = rng.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True) + 1e-12
    r = radius + rng.normal(0.0, jitter, size=(n, 1))
    return center + d * r


def _surface_points(rng, n, surf, n_surf=3):
    """Points on `n_surf` seeded Gaussian-perturbed spheres (|p|_inf <= 0.3)."""
    idx = rng.integers(0, n_surf, size=n)
    c = surf[0][idx]
    r = surf[1][idx][:, None]
    return c + _unit(rng, n) * (r + rng.normal(0.0, 0.01, (n, 1)))


def _unit(rng, n):
    d = rng.standard_normal((n, 3))
    return d / (np.linalg.norm(d, axis=1, keepdims=True) + 1e-12)


def _shell_points(rng, n, inner=0.36):
    """Points uniform in the cube shell inner < |p|_inf < 0.5."""
    pts = []
    got = 0
    while got < n:
        p = rng.uniform(-0.5, 0.5, size=(2 * n + 1024, 3))
        p = p[np.abs(p).max(1) > inner]
        pts.append(p)
        got += len(p)
    return np.concatenate(pts, 0)[:n]


def _region_levels(pts, l0, l1, salt):
    """Level of each point, constant over level-l0 regions (so cells never overlap)."""
    if l0 == l1:
        return np.full(len(pts), l0, np.int64)
    side = 1 << l0
    rid = np.clip(np.floor((pts + 0.5) * side).astype(np.int64), 0, side - 1)
    h = (rid[:, 0] * 73856093) ^ (rid[:, 1] * 19349663) ^ (rid[:, 2] * 83492791) ^ (salt * 2654435761)
    h = (h ^ (h >> 13)) * 0x5bd1e995
    h = (h ^ (h >> 15)) & 0x7fffffff
    return l0 + h % (l1 - l0 + 1)


def _take(rng, arr, n):
    if len(arr) <= n:
        return arr
    return np.sort(rng.choice(arr, size=n, replace=False))


def make_voxels(n, seed, kind="sphere", surf_levels=(6, 8), bg_levels=(5, 7), surf_frac=0.7):
    """Octree voxels: kind='sphere' (jittered sphere shell of radius 0.4) or
    'mixed' (three surfaces + background shell).  Levels are drawn per
    coarse region, so no voxel is an ancestor of another.
    Returns (octpath int64 [N], level int8 [N])."""
    rng = np.random.default_rng(seed)
    if kind == "sphere":
        groups = [("sphere", n, surf_levels)]
    else:
        n_s = int(round(n * surf_frac))
        # Background first: its level range may hold fewer cells than asked
        # for, and the surfaces then make up the difference.
        groups = [("bg", n - n_s, bg_levels), ("surf", n_s, surf_levels)]
    surf = (rng.uniform(-0.08, 0.08, size=(3, 3)), rng.uniform(0.1, 0.18, size=3))
    all_ijk, all_lv = [], []
    deficit = 0
    for gi, (name, cnt, (l0, l1)) in enumerate(groups):
        cnt += deficit
        keys = np.zeros(0, np.int64)
        m = max(4096, int(cnt * 1.3))
        for _ in range(10):
            if name == "sphere":
                pts = _sphere_points(rng, m, np.zeros(3), 0.4, 0.02)
            elif name == "surf":
                pts = _surface_points(rng, m, surf)
            else:
                pts = _shell_points(rng, m)
            pts = np.clip(pts, -0.5 + 1e-7, 0.5 - 1e-7)
            lv = _region_levels(pts, l0, l1, seed * 7 + gi)
            ijk = _cells_from_points(pts, lv)
            before = len(keys)
            keys = np.unique(np.concatenate([keys, _cell_key(ijk, lv)]))
            if len(keys) >= cnt or len(keys) < before * 1.02:
                break  # enough cells, or the level range is saturated
            m = min(int(m * 1.5), 4 * cnt + 4096)
        keys = _take(rng, keys, cnt)
        deficit = cnt - len(keys)
        lv = keys >> 52
        idx = keys & ((np.int64(1) << 52) - 1)
        side = np.left_shift(np.int64(1), lv)
        ijk = np.stack([idx // (side * side), (idx // side) % side, idx % side], 1)
        all_ijk.append(ijk)
        all_lv.append(lv)
    ijk = np.concatenate(all_ijk, 0)
    lv = np.concatenate(all_lv, 0)
    if len(groups) > 1:
        keep = remove_overlaps(ijk, lv)
        ijk, lv = ijk[keep], lv[keep]
    perm = rng.permutation(len(lv))
    ijk, lv = ijk[perm], lv[perm]
    return ijk_to_octpath(ijk, lv), lv.astype(np.int8)


def look_at(position, target=(0.0, 0.0, 0.0), up=(0.0, -1.0, 0.0)):
    """OpenCV-convention (x right, y down, z forward) camera -> (w2c, c2w) float32 4x4."""
    pos = np.asarray(position, np.float64)
    fwd = np.asarray(target, np.float64) - pos
    fwd /= np.linalg.norm(fwd)
    upv = np.asarray(up, np.float64)
    right = np.cross(fwd, upv)
    if np.linalg.norm(right) < 1e-6:
        right = np.cross(fwd, np.array([1.0, 0.0, 0.0]))
    right /= np.linalg.norm(right)
    down = np.cross(fwd, right)
    c2w = np.eye(4)
    c2w[:3, 0], c2w[:3, 1], c2w[:3, 2], c2w[:3, 3] = right, down, fwd, pos
    w2c = np.linalg.inv(c2w)
    return w2c.astype(np.float32), c2w.astype(np.float32)


@dataclass
class Camera:
    width: int
    height: int
    tanfovx: float
    tanfovy: float
    cx: float
    cy: float
    w2c: np.ndarray
    c2w: np.ndarray
    near: float = 0.02

    @property
    def position(self):
        return self.c2w[:3, 3]


def make_camera(width, height, fovx_deg, position, target=(0.0, 0.0, 0.0)):
    w2c, c2w = look_at(position, target)
    tanfovx = math.tan(math.radians(fovx_deg) * 0.5)
    tanfovy = tanfovx * height / width
    return Camera(int(width), int(height), tanfovx, tanfovy, width * 0.5, height * 0.5, w2c, c2w)


def orbit_cameras(n, seed, radius=(2.0, 4.0), size_range=((640, 480), (1600, 1200)), fovx_deg=50.0,
                  hemisphere=False, fixed_size=None):
    rng = np.random.default_rng(seed)
    cams = []
    for _ in range(n):
        d = rng.standard_normal(3)
        if hemisphere:
            d[1] = -abs(d[1])  # y is down in the world frame used here: upper hemisphere
        d /= np.linalg.norm(d)
        r = rng.uniform(*radius)
        if fixed_size is not None:
            w, h = fixed_size
        else:
            w = int(rng.integers(size_range[0][0], size_range[1][0] + 1))
            h = int(rng.integers(size_range[0][1], size_range[1][1] + 1))
        cams.append(make_camera(w, h, fovx_deg, d * r))
    return cams


@dataclass
class Scene:
    name: str
    octpath: np.ndarray
    octlevel: np.ndarray
    centers: np.ndarray
    lengths: np.ndarray
    geos: np.ndarray
    sh0: np.ndarray
    shs: np.ndarray
    cameras: list
    targets: list = field(default_factory=list)

    @property
    def n_voxels(self):
        return len(self.octpath)

    @property
    def max_level(self):
        return int(self.octlevel.max()) if len(self.octlevel) else 0


def _params(rng, n, geo_mu, geo_sigma, sh_sigma=0.2, sh_deg=3):
    geos = rng.normal(geo_mu, geo_sigma, size=(n, 8)).astype(np.float32)
    m = (sh_deg + 1) ** 2
    sh0 = rng.normal(0.0, sh_sigma, size=(n, 3)).astype(np.float32)
    shs = rng.normal(0.0, sh_sigma, size=(n, m - 1, 3)).astype(np.float32)
    return geos, sh0, shs


def build_scene(name, n_voxels, seed, kind, surf_levels, bg_levels, geo_mu, geo_sigma, cameras, n_targets=1):
    path, lv = make_voxels(n_voxels, seed, kind, surf_levels, bg_levels)
    centers, lengths = decode_voxels(path, lv)
    rng = np.random.default_rng(seed + 1)
    geos, sh0, shs = _params(rng, len(path), geo_mu, geo_sigma)
    trng = np.random.default_rng(seed + 2)
    targets = [trng.uniform(0.0, 1.0, size=(3, c.height, c.width)).astype(np.float32) for c in cameras[:n_targets]]
    return Scene(name, path, lv, centers, lengths, geos, sh0, shs, cameras, targets)


def _unit_dir(rng):
    d = rng.standard_normal(3)
    return d / np.linalg.norm(d)


def config_cameras(name, seed=0, view_set=0):
    """Cameras of a benchmark configuration (see config_scene).  view_set 0
    is the configuration's own set; view_set k > 0 draws another set of the
    same count, sizes and distance distribution (the views of rank k in a
    view-parallel run, so every rank does the single-GPU amount of work)."""
    rng = np.random.default_rng(seed + 7919 * view_set)
    if name == "c1":
        if view_set == 0:
            d1 = np.array([0.9, -0.7, -1.0]) / np.linalg.norm([0.9, -0.7, -1.0])
            return [make_camera(256, 256, 50.0, (0.0, 0.0, -1.5)), make_camera(256, 256, 50.0, d1 * 1.5),
                    # inside the sphere shell: voxels straddle the camera's axis planes (multi-quadrant)
                    make_camera(200, 136, 70.0, (0.03, -0.02, 0.01), target=(0.4, 0.1, 0.3))]
        return [make_camera(256, 256, 50.0, _unit_dir(rng) * 1.5), make_camera(256, 256, 50.0, _unit_dir(rng) * 1.5),
                make_camera(200, 136, 70.0, _unit_dir(rng) * 0.03, target=_unit_dir(rng) * 0.5)]
    if name == "c2":
        d = np.array([0.6, -0.5, -1.2]) if view_set == 0 else _unit_dir(rng)
        return [make_camera(1297, 840, 50.0, d / np.linalg.norm(d) * 1.6)]
    if name == "c3":
        return orbit_cameras(16, seed + 10 + 7919 * view_set)
    if name == "c4":
        return orbit_cameras(8, seed + 20 + 7919 * view_set, radius=(1.5, 2.0), fixed_size=(1920, 1080))
    if name == "c5":
        rng = np.random.default_rng(seed + 30 + 7919 * view_set)
        cams = []
        for _ in range(32):
            sc = rng.uniform(0.5, 1.0)
            cams += orbit_cameras(1, int(rng.integers(1 << 30)), radius=(1.5, 2.5), hemisphere=True,
                                  fixed_size=(int(1920 * sc) // 2 * 2, int(1080 * sc) // 2 * 2))
        return cams
    raise ValueError(f"unknown config {name}")


def config_scene(name, seed=0, n_voxels=None):
    """Synthetic stand-ins for the five benchmark configurations.

    c1: 20k voxels, levels 6-8 on a jittered sphere (r=0.4), geos~N(-1,1),
        256x256 fov 50 deg at distance 1.5 (+ a second generic camera, and a
        200x136 camera inside the shell for multi-quadrant coverage).
    c2: 2M voxels, 70% on three Gaussian-perturbed surfaces (levels 8-12),
        30% in a background shell (levels 5-7), geos~N(-2,1.5), one 1297x840 view.
    c3: the c2 scene seen by 16 orbit cameras (radius 2-4, 640x480..1600x1200).
    c4: 8M voxels (levels 8-14, same mix), 8 views at 1920x1080.
    c5: 16M voxels (levels 6-16), 32 views 960x540..1920x1080 on a hemisphere.
    `n_voxels` overrides the voxel count (for scaled-down tests).
    """
    cams = config_cameras(name, seed)
    if name == "c1":
        return build_scene("c1", n_voxels or 20000, seed, "sphere", (6, 8), (6, 8), -1.0, 1.0, cams)
    if name in ("c2", "c3"):
        return build_scene(name, n_voxels or 2_000_000, seed, "mixed", (8, 12), (5, 7), -2.0, 1.5, cams)
    if name == "c4":
        return build_scene("c4", n_voxels or 8_000_000, seed, "mixed", (8, 14), (5, 7), -2.0, 1.5, cams)
    return build_scene("c5", n_voxels or 16_000_000, seed, "mixed", (6, 16), (5, 7), -2.0, 1.5, cams)


def grid_keys(octpath, level, dev):
    """Corner-point indices [N,8] of octree voxels into a deduplicated grid.

    Corner (i+di, j+dj, k+dk) of a level-l cell is expressed at the finest
    level (shifted by 16-l) so coincident corners of cells of different sizes
    share one grid point; corner order is di*4 + dj*2 + dk.  Returns
    (vox_key int64[N,8] on `dev`, number of grid points).
    """
    import torch
    ijk = torch.from_numpy(octpath_to_ijk(octpath, level)).to(dev)
    shift = (16 - torch.from_numpy(np.asarray(level, dtype=np.int64).reshape(-1))).to(dev)
    off = torch.tensor([[(c >> 2) & 1, (c >> 1) & 1, c & 1] for c in range(8)], dtype=torch.int64, device=dev)
    corner = (ijk[:, None, :] + off[None]) << shift[:, None, None]
    code = (corner[..., 0] << 34) | (corner[..., 1] << 17) | corner[..., 2]
    uniq, inv = torch.unique(code.reshape(-1), return_inverse=True)
    return inv.reshape(-1, 8).contiguous(), int(uniq.numel())


def grid_params(sc, dev, seed=0):
    """Grid-point parametrisation of a scene's densities, as the reference
    trains them (sparse_voxel_gears/constructor.py:71-73): vox_key int64
    [P,8] on `dev` (grid_keys) and seeded grid values [M] drawn from the
    scene's density distribution (the mean and spread of its per-voxel
    corner values).  Returns (vox_key, grid_pts numpy fp32)."""
    key, M = grid_keys(sc.octpath, sc.octlevel, dev)
    rng = np.random.default_rng(seed + 5)
    mu, sd = float(np.mean(sc.geos)), float(np.std(sc.geos))
    return key, rng.normal(mu, sd, size=M).astype(np.float32)


def deep_scene(n_voxels=20000, n_chains=64, seed=0, max_levels=21):
    """An octree 21 levels deep (the new_cuda backend's depth): the c1 sphere
    scene (levels 6-8) with `n_chains` of its voxels refined down to level 21
    along a seeded path -- at every level 7 of the 8 children are kept and one
    is refined further -- so every level from 6 to 21 holds voxels and their
    63-bit Morton ranks differ below the 48 bits a 16-level octree uses.
    No voxel is an ancestor of another.  Octree paths use the 21-level
    encoding (utils.cu:129-158 with MAX_NUM_LEVELS = 21)."""
    base = config_scene("c1", seed=seed, n_voxels=n_voxels)
    ijk = octpath_to_ijk(base.octpath, base.octlevel)
    lv = base.octlevel.astype(np.int64)
    rng = np.random.default_rng(seed + 77)
    pick = rng.choice(len(lv), size=min(n_chains, len(lv)), replace=False)
    keep = np.ones(len(lv), bool)
    keep[pick] = False
    cells, levels = [ijk[keep]], [lv[keep]]
    offs = np.array([[(c >> 2) & 1, (c >> 1) & 1, c & 1] for c in range(8)], np.int64)
    for p in pick:
        cur, l = ijk[p], int(lv[p])
        while l < max_levels:
            kids = 2 * cur[None, :] + offs
            nxt = int(rng.integers(8))
            cells.append(np.delete(kids, nxt, axis=0))
            levels.append(np.full(7, l + 1, np.int64))
            cur, l = kids[nxt], l + 1
        cells.append(cur[None, :])
        levels.append(np.array([l], np.int64))
    ijk, lv = np.concatenate(cells), np.concatenate(levels)
    path = ijk_to_octpath(ijk, lv, max_levels)
    centers, lengths = decode_voxels(path, lv, max_levels)
    geos, sh0, shs = _params(np.random.default_rng(seed + 1), len(path), -1.0, 1.0)
    return Scene("deep", path, lv.astype(np.int8), centers, lengths, geos, sh0, shs, config_cameras("c1", seed))


def scene_cache_dir():
    """Directory of cached scenes: SVR_SCENE_CACHE, else a per-user cache
    directory (created private to the user)."""
    return os.environ.get("SVR_SCENE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "sv_raster_b200",
                                                              "scenes")


def generator_digest():
    """Short digest of this module's source: cached scenes are keyed by it, so
    a change to the generator never reuses scenes an older one built."""
    import hashlib
    with open(os.path.abspath(__file__), "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()[:12]


def cached_scene_path(name, seed=0, n_voxels=None):
    """Cache file of a configuration's scene for the current generator."""
    return os.path.join(scene_cache_dir(), f"{name}_{seed}_{n_voxels or 0}_{generator_digest()}.pkl")


def cached_config_scene(name, seed=0, n_voxels=None):
    """config_scene with an on-disk cache (the 8M- and 16M-voxel scenes take
    minutes to build on the CPU).  Scenes are deterministic in (name, seed,
    n_voxels) for a given generator source (its digest is part of the file
    name), so a cached copy equals a rebuilt one; the cache directory is
    the user's own, never a shared temporary directory, because entries are
    unpickled.  Writers use a per-process temporary name, so concurrent ranks
    building the same scene do not interleave their writes."""
    path = cached_scene_path(name, seed, n_voxels)
    d = os.path.dirname(path)
    if os.path.exists(path):
        try:
            with open(path, "rb") as f:
                return pickle.load(f)
        except Exception:
            pass  # unreadable or partial entry: rebuild it
    sc = config_scene(name, seed=seed, n_voxels=n_voxels)
    try:
        os.makedirs(d, mode=0o700, exist_ok=True)
        tmp = f"{path}.{os.getpid()}.tmp"
        with open(tmp, "wb") as f:
            pickle.dump(sc, f, protocol=4)
        os.replace(tmp, path)
    except OSError:
        pass
    return sc
