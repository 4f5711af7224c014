"""Gradient and precision checks at scale.

* C2 scene (2M voxels): GPU fp32 analytic gradients of a random linear
  function of (colour, T) against FP64 central differences of the FP64 oracle
  on 256 randomly chosen visible voxels.  The view is a 96x96 window of the
  1297x840 camera (same focal length, shifted principal point), so each FD
  evaluation re-composites only that window; projection and binning do not
  depend on the perturbed parameters and are reused.
* bf16 storage (densities and SH in bf16, fp32 compositing): rendered PSNR
  against a target within 0.01 dB of the FP64 oracle's, and the gradient's
  relative error against the fp32 path, on a window of a c4-like view.
"""
import math

import numpy as np
import pytest
import torch

import oracle as O
from sv_raster_b200 import _C as mC
from sv_raster_b200 import synthetic
from sv_raster_b200.batched import BatchedRasterizer, BatchedRender

pytestmark = pytest.mark.gpu


def window(cam, x0, y0, w, h):
    """Camera restricted to the pixel window [x0, x0+w) x [y0, y0+h)."""
    c = synthetic.Camera(w, h, cam.tanfovx * w / cam.width, cam.tanfovy * h / cam.height, cam.cx - x0, cam.cy - y0,
                         cam.w2c, cam.c2w, cam.near)
    return c


def _gpu_grads(sc, cam, geos, rgbs, wC, wT):
    t = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dt)
    octpath, centers, lengths = t(sc.octpath.reshape(-1, 1), torch.int64), t(sc.centers), t(sc.lengths)
    w2c, c2w = t(cam.w2c), t(cam.c2w)
    nd, geom = mC.rasterize_preprocess(cam.width, cam.height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w,
                                       cam.near, octpath, centers, lengths)
    g, r = t(geos), t(rgbs)
    out = mC.rasterize_voxels(1, cam.width, cam.height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, 0.0,
                              False, False, False, False, octpath, centers, lengths, g, r, geom)
    e = torch.empty(0, device="cuda")
    grads = mC.rasterize_voxels_backward(out[0], 1, cam.width, cam.height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy,
                                         w2c, c2w, 0.0, octpath, centers, lengths, g, r, geom, out[1], out[2],
                                         out[6], t(wC), e, e, t(wT[None]), 0.0, e, 0.0, 0.0, False, False, out[4],
                                         out[5])
    return out[3].cpu().numpy(), grads[0].cpu().numpy(), grads[1].cpu().numpy()


def test_c2_gradients_match_fp64_central_differences():
    sc = synthetic.config_scene("c2")
    full = sc.cameras[0]
    cam = window(full, 600, 380, 96, 96)
    rng = np.random.default_rng(21)
    rgbs = rng.uniform(0.05, 0.95, size=(sc.n_voxels, 3)).astype(np.float32)
    wC = rng.standard_normal((3, cam.height, cam.width)).astype(np.float32)
    wT = rng.standard_normal((cam.height, cam.width)).astype(np.float32)
    color, dgeo, drgb = _gpu_grads(sc, cam, sc.geos, rgbs, wC, wT)
    # FP64 oracle: projection + binning once
    ndup, bbox, quad = O.preprocess(cam, sc.centers, sc.lengths)
    keys, vals, ranges = O.binning(cam, sc.octpath, ndup, bbox, quad)

    def loss(geos, rg):
        o = O.render_fwd(cam, ranges, vals, bbox, sc.centers, sc.lengths, geos, rg, mode="f64")
        return float((o["color"] * wC).sum() + (o["T"] * wT).sum()), o

    L0, o0 = loss(sc.geos, rgbs)
    assert np.abs(o0["color"] - color).max() < 1e-4
    cand = np.where(np.abs(dgeo).sum(1) > 0)[0]
    assert len(cand) >= 256, len(cand)
    pick = rng.choice(cand, size=256, replace=False)
    num, ana = [], []
    eps = 1e-3
    for v in pick:
        c = int(rng.integers(0, 8))
        gp, gm = sc.geos.copy(), sc.geos.copy()
        gp[v, c] += eps
        gm[v, c] -= eps
        h = float(gp[v, c]) - float(gm[v, c])
        num.append((loss(gp, rgbs)[0] - loss(gm, rgbs)[0]) / h)
        ana.append(dgeo[v, c])
        k = int(rng.integers(0, 3))
        rp, rm = rgbs.copy(), rgbs.copy()
        rp[v, k] += eps
        rm[v, k] -= eps
        h = float(rp[v, k]) - float(rm[v, k])
        num.append((loss(sc.geos, rp)[0] - loss(sc.geos, rm)[0]) / h)
        ana.append(drgb[v, k])
    num, ana = np.array(num), np.array(ana)
    rel = float(np.linalg.norm(num - ana) / np.linalg.norm(num))
    print(f"C2 FD check: 256 voxels, 512 partials, relative error {rel:.3e}")
    assert rel < 1e-3


def _psnr(a, b):
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return 10 * math.log10(1.0 / max(mse, 1e-30))


class _DevCam:
    def __init__(self, c):
        self.width, self.height = c.width, c.height
        self.tanfovx, self.tanfovy, self.cx, self.cy, self.near = c.tanfovx, c.tanfovy, c.cx, c.cy, c.near
        self.w2c = torch.from_numpy(c.w2c).cuda()
        self.c2w = torch.from_numpy(c.c2w).cuda()


def test_bf16_storage_precision_c4_window():
    sc = synthetic.config_scene("c4", n_voxels=1_000_000)
    cam = window(sc.cameras[0], 900, 500, 160, 120)
    t = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dt)
    octpath, centers, lengths = t(sc.octpath.reshape(-1, 1), torch.int64), t(sc.centers), t(sc.lengths)
    geos32, sh032, shs32 = t(sc.geos), t(sc.sh0), t(sc.shs)
    tgt = np.random.default_rng(5).uniform(0, 1, (3, cam.height, cam.width)).astype(np.float32)
    res = {}
    for name, dt in (("fp32", torch.float32), ("bf16", torch.bfloat16)):
        r = BatchedRasterizer([_DevCam(cam)], octpath, centers, lengths, max_level=sc.max_level)
        geos = geos32.detach().to(dt).clone().requires_grad_(True)
        sh0 = sh032.detach().to(dt).clone().requires_grad_(True)
        shs = shs32.detach().to(dt).clone().requires_grad_(True)
        r.fit_capacity(sh0.detach(), shs.detach(), 3)
        color, T = BatchedRender.apply(r, 3, geos, sh0, shs)
        loss = ((color.view(3, cam.height, cam.width) - t(tgt)) ** 2).mean()
        loss.backward()
        res[name] = (color.detach().view(3, cam.height, cam.width).cpu().numpy(), geos.grad.float().cpu().numpy(),
                     shs.grad.float().cpu().numpy())
    # FP64 oracle on the original (fp32) parameters
    rgbs64 = O.sh_fwd(3, np.arange(sc.n_voxels), sc.centers, cam.position, sc.sh0, sc.shs, mode="f64")
    o = O.render_view(cam, sc.octpath, sc.centers, sc.lengths, sc.geos, rgbs64.astype(np.float32), mode="f64")
    p64 = _psnr(o["color"], tgt)
    p32, p16 = _psnr(res["fp32"][0], tgt), _psnr(res["bf16"][0], tgt)
    img_err16 = float(np.abs(res["bf16"][0] - o["color"]).max())
    gref = res["fp32"][1]
    g_rel = float(np.linalg.norm(res["bf16"][1] - gref) / np.linalg.norm(gref))
    s_rel = float(np.linalg.norm(res["bf16"][2] - res["fp32"][2]) / np.linalg.norm(res["fp32"][2]))
    print(f"PSNR vs target: fp64 oracle {p64:.4f} dB, fp32 {p32:.4f} dB, bf16 storage {p16:.4f} dB; "
          f"bf16 image max err vs fp64 {img_err16:.2e}; density grad rel err bf16 vs fp32 {g_rel:.2e}; "
          f"SH grad rel err {s_rel:.2e}")
    assert abs(p32 - p64) < 1e-3
    assert abs(p16 - p64) < 0.01
    assert g_rel < 0.05 and s_rel < 0.05
