"""Error of GPU images and gradients against the FP64 compositing oracle on a
seeded sample of full 16x16 tiles -- TEST / MEASUREMENT INFRASTRUCTURE.

Used by the precision tests and by bench.py's baseline leg (outside every
timed region).  The oracle (svr_oracle.c in FP64 mode) projects and bins the
view in fp32 exactly as the reference does (preprocess.cu:24-132,
forward.cu:518-598), evaluates SH in FP64 (sh_compute.cu:54-176) and
composites and back-propagates the sampled tiles in FP64 (forward.cu:39-392,
backward.cu:35-530).

Gradients are compared for the same upstream gradient on both sides: the
caller's dL/dcolour restricted to the sampled tiles (zero elsewhere), so only
the sampled pixels contribute to either side's parameter gradients.
"""
import math

import numpy as np

import oracle as O

TILE = 16


def tile_runs(cam, n_runs=64, run_len=16, seed=0):
    """Seeded, disjoint runs [lo, hi) of consecutive tile indices (row-major 16x16 tiles)."""
    gx, gy = (cam.width + TILE - 1) // TILE, (cam.height + TILE - 1) // TILE
    T = gx * gy
    if n_runs * run_len >= T:
        return [(0, T)]
    rng = np.random.default_rng(seed)
    slots = rng.choice(T // run_len, size=n_runs, replace=False)
    return sorted((int(s) * run_len, int(s) * run_len + run_len) for s in slots)


def tile_mask(cam, runs):
    """[H, W] bool mask of the pixels of the sampled tiles."""
    gx = (cam.width + TILE - 1) // TILE
    m = np.zeros((cam.height, cam.width), bool)
    for lo, hi in runs:
        for t in range(lo, hi):
            ty, tx = divmod(t, gx)
            m[ty * TILE:(ty + 1) * TILE, tx * TILE:(tx + 1) * TILE] = True
    return m


def psnr(a, b, mask):
    """PSNR (peak 1) of colour images [3,H,W] over the masked pixels."""
    d = (np.asarray(a, np.float64) - np.asarray(b, np.float64))[:, mask]
    mse = float(np.mean(d * d))
    return 10.0 * math.log10(1.0 / max(mse, 1e-30))


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


class OracleView:
    """FP64 oracle forward of the sampled tiles of one view of a scene (fp32
    master parameters), and its backward for a given upstream gradient."""

    def __init__(self, sc, cam, runs, sh_degree=3):
        self.sc, self.cam, self.runs = sc, cam, runs
        self.mask = tile_mask(cam, runs)
        self.ndup, self.bbox, self.quad = O.preprocess(cam, sc.centers, sc.lengths)
        _, self.vals, self.ranges = O.binning(cam, sc.octpath, self.ndup, self.bbox, self.quad)
        self.vis = np.nonzero(self.ndup)[0]
        self.sh_degree = sh_degree
        self.rgbs64 = O.sh_fwd(sh_degree, self.vis, sc.centers, cam.position, sc.sh0, sc.shs, mode="f64")
        H, W = cam.height, cam.width
        gx, gy = (W + TILE - 1) // TILE, (H + TILE - 1) // TILE
        self.color = np.zeros((3, H, W))
        self.T = np.zeros((H, W))
        self.n_contrib = np.zeros((H, W), np.uint32)
        self.tile_last = np.zeros(gx * gy, np.uint32)
        for lo, hi in runs:
            o = O.render_fwd(cam, self.ranges, self.vals, self.bbox, sc.centers, sc.lengths, sc.geos, self.rgbs64,
                             mode="f64", tiles=(lo, hi))
            self.color[:, self.mask] += o["color"][:, self.mask]
            self.T[self.mask] += o["T"][self.mask]
            self.n_contrib[self.mask] |= o["n_contrib"][self.mask]
            self.tile_last[lo:hi] = o["tile_last"][lo:hi]

    def backward(self, dL_dcolor):
        """FP64 (dL_dgeos [P,8], dL_dsh0 [P,3], dL_dshs [P,M-1,3]) for the upstream
        gradient restricted to the sampled tiles."""
        sc, cam = self.sc, self.cam
        dC = np.where(self.mask[None], np.asarray(dL_dcolor, np.float32), 0.0).astype(np.float32)
        dT = np.zeros((cam.height, cam.width), np.float32)
        P = sc.n_voxels
        dgeo = np.zeros((P, 8))
        drgb = np.zeros((P, 3))
        for lo, hi in self.runs:
            g = O.render_bwd(cam, self.ranges, self.tile_last, self.vals, self.bbox, sc.centers, sc.lengths, sc.geos,
                             self.rgbs64, self.n_contrib, self.T, dC, dT, mode="f64", tiles=(lo, hi))
            dgeo += g["dL_dgeos"]
            drgb += g["dL_drgbs"]
        M = 1 + sc.shs.shape[1]
        dsh0, dshs = O.sh_bwd(self.sh_degree, M, self.vis, sc.centers, cam.position, drgb, mode="f64")
        return dgeo, dsh0, dshs


def report(orc, target, images, grads, dC):
    """Errors of named GPU images ({name: [3,H,W]}) and gradients ({name:
    (dgeo, dsh0, dshs)}, computed for the masked upstream gradient dC) against
    the oracle.  Returns a JSON-able dict."""
    m = orc.mask
    p64 = psnr(orc.color, target, m)
    out = {"tiles": int(sum(hi - lo for lo, hi in orc.runs)), "pixels": int(m.sum()),
           "psnr_fp64_oracle_db": round(p64, 4)}
    for name, img in images.items():
        img = np.asarray(img, np.float64)
        d = np.abs(img[:, m] - orc.color[:, m])
        out[name] = {"psnr_db": round(psnr(img, target, m), 4), "psnr_delta_db": round(psnr(img, target, m) - p64, 5),
                     "image_max_abs_err": float(f"{d.max():.3e}"),
                     "image_rel_err": float(f"{rel(img[:, m], orc.color[:, m]):.3e}")}
    if grads:
        gdgeo, gdsh0, gdshs = orc.backward(dC)
        for name, (dgeo, dsh0, dshs) in grads.items():
            out.setdefault(name, {})
            out[name].update({"dL_dgeos_rel_err": float(f"{rel(dgeo, gdgeo):.3e}"),
                              "dL_dsh0_rel_err": float(f"{rel(dsh0, gdsh0):.3e}"),
                              "dL_dshs_rel_err": float(f"{rel(dshs, gdshs):.3e}")})
    return out


class _DevCam:
    def __init__(self, c, dev):
        import torch
        self.width, self.height = c.width, c.height
        self.tanfovx, self.tanfovy, self.cx, self.cy, self.near = c.tanfovx, c.tanfovy, c.cx, c.cy, c.near
        self.w2c = torch.from_numpy(np.ascontiguousarray(c.w2c)).to(dev)
        self.c2w = torch.from_numpy(np.ascontiguousarray(c.c2w)).to(dev)


def gpu_view(sc, cam, target, mask, dev="cuda", tile_size=8):
    """One view through the native paths: the batched path with bf16 storage of
    densities and SH, and the plain fp32 path.  The upstream gradient is the
    batched image's L2-loss gradient against `target`, restricted to `mask`,
    and both backward passes use it.  Returns (images, grads, dC) as numpy."""
    import torch

    from sv_raster_b200 import _C as mC
    from sv_raster_b200.batched import BatchedRasterizer
    t = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dt)
    octpath, centers, lengths = t(sc.octpath.reshape(-1), torch.int64), t(sc.centers), t(sc.lengths)
    H, W = cam.height, cam.width
    M = 1 + sc.shs.shape[1]
    geos16, sh016, shs16 = (t(sc.geos).to(torch.bfloat16).contiguous(), t(sc.sh0).to(torch.bfloat16).contiguous(),
                            t(sc.shs).to(torch.bfloat16).contiguous())
    r = BatchedRasterizer([_DevCam(cam, dev)], octpath, centers, lengths, max_level=sc.max_level, tile_size=tile_size)
    r.fit_capacity(sh016, shs16, 3)
    r.prepare(sh016, shs16, 3)
    color16, T16 = r.render(geos16)
    dC = (2.0 / (3 * H * W)) * (color16.view(3, H, W) - t(target)) * t(mask)[None]
    dC = dC.contiguous()
    g16 = r.backward(geos16, T16, dC.reshape(-1), torch.zeros_like(T16), 3, M)
    images = {"batched_bf16": color16.view(3, H, W).cpu().numpy()}
    grads = {"batched_bf16": (g16[0].cpu().numpy(), g16[2].cpu().numpy(), g16[3].cpu().numpy())}
    del r, geos16, sh016, shs16, g16
    # plain fp32 path, the reference's call sequence (renderer.py:66-248)
    w2c, c2w = t(cam.w2c), t(cam.c2w)
    geos, sh0, shs = t(sc.geos), t(sc.sh0), t(sc.shs)
    op = octpath.view(-1, 1)
    ndup, geom = mC.rasterize_preprocess(W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, cam.near, op,
                                         centers, lengths)
    vis = torch.nonzero(ndup > 0).reshape(-1)
    pos = c2w[:3, 3].contiguous()
    rgbs = mC.sh_compute(3, vis, centers, pos, sh0, shs)
    out = mC.rasterize_voxels(1, W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, 0.0, False, False, False,
                              False, op, centers, lengths, geos, rgbs, geom)
    e = torch.empty(0, device=dev)
    g = mC.rasterize_voxels_backward(out[0], 1, W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, 0.0, op,
                                     centers, lengths, geos, rgbs, geom, out[1], out[2], out[6], dC, e, e,
                                     torch.zeros_like(out[6]), 0.0, e, 0.0, 0.0, False, False, out[4], out[5])
    d0, ds = mC.sh_compute_bw(3, M, vis, centers, pos, rgbs, g[1])
    images["plain_fp32"] = out[3].cpu().numpy()
    grads["plain_fp32"] = (g[0].cpu().numpy(), d0.cpu().numpy(), ds.cpu().numpy())
    return images, grads, dC.cpu().numpy()


def measure(sc, cam, target, runs=None, dev="cuda"):
    """Errors of the batched bf16-storage and plain fp32 paths on one view
    against the FP64 oracle over the sampled tiles (all tiles if runs is
    'all').  Returns the report dict."""
    if runs is None:
        runs = tile_runs(cam)
    elif runs == "all":
        gx, gy = (cam.width + TILE - 1) // TILE, (cam.height + TILE - 1) // TILE
        runs = [(0, gx * gy)]
    mask = tile_mask(cam, runs)
    images, grads, dC = gpu_view(sc, cam, target, mask.astype(np.float32), dev)
    orc = OracleView(sc, cam, runs)
    rep = report(orc, target, images, grads, dC)
    rep["oracle_params"] = "fp32 master parameters (the bf16 path's error includes its storage rounding)"
    return rep
