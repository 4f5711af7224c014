"""The CUDA path against the golden vectors of the reference backend
(tests/golden/*.npz): integers bit-exact, images and transmittance bitwise
equal (same fp32 arithmetic as the reference), gradients within 1e-5
relative (atomic summation order differs)."""
import glob
import os

import numpy as np
import pytest
import torch

from conftest import ROOT
from refutil import SceneTensors
from sv_raster_b200 import _C as mC
from sv_raster_b200 import synthetic

pytestmark = pytest.mark.gpu
GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz")))


@pytest.fixture(scope="module")
def c1():
    return SceneTensors(synthetic.config_scene("c1"))


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_cuda_path_matches_reference_goldens(c1, path):
    import make_golden
    g = np.load(path)
    ci = int(g["camera"])
    ns = int(g["n_samp"])
    depth, dist, normal, maxw = [bool(x) for x in g["flags"]]
    bg = float(g["bg"])
    lR, lA, lD = [float(x) for x in g["lambdas"]]
    cam, w2c, c2w = c1.cam(ci)
    W, H = cam.width, cam.height
    P = c1.centers.shape[0]
    ndup, geom = mC.rasterize_preprocess(W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, cam.near,
                                         c1.octpath, c1.centers, c1.lengths)
    assert np.array_equal(ndup.cpu().numpy(), g["n_dup"])
    vis = torch.where(ndup > 0)[0]
    assert np.array_equal(vis.cpu().numpy(), g["visible"])
    _, _, bb, qd = mC.unpack_geom_state(geom, P)
    assert np.array_equal(bb[vis].cpu().numpy(), g["bbox"])
    assert np.array_equal(qd[vis].cpu().numpy(), g["quad"])
    rgbs = mC.sh_compute(3, vis, c1.centers, c2w[:3, 3].contiguous(), c1.sh0, c1.shs)
    assert np.array_equal(rgbs.cpu().numpy(), g["rgbs"])
    out = mC.rasterize_voxels(ns, W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, bg, depth, dist, normal,
                              maxw, c1.octpath, c1.centers, c1.lengths, c1.geos, rgbs, geom)
    R, binning, img, color, odepth, onormal, T, max_w = out
    assert R == int(g["num_rendered"])
    k, v = mC.unpack_sorted_list(binning, R, W, H)
    assert np.array_equal(k.cpu().numpy(), g["keys"])
    assert np.array_equal(v.cpu().numpy(), g["vals"])
    ranges, tile_last, n_contrib = mC.unpack_ImageState(W, H, img)
    assert np.array_equal(ranges.cpu().numpy(), g["ranges"])
    assert np.array_equal(tile_last.cpu().numpy(), g["tile_last"])
    assert np.array_equal(n_contrib.cpu().numpy(), g["n_contrib"])
    assert np.array_equal(color.cpu().numpy(), g["color"])
    assert np.array_equal(T.cpu().numpy(), g["T"])
    if depth or dist:
        assert np.abs(odepth.cpu().numpy() - g["depth"]).max() < 1e-6
    if normal:
        assert np.abs(onormal.cpu().numpy() - g["normal"]).max() < 1e-6
    if maxw:
        assert np.array_equal(max_w.cpu().numpy(), g["max_w"])
    up = make_golden.upstream(ci, H, W)
    t = lambda a: torch.from_numpy(a).cuda()
    e = torch.empty(0, device="cuda")
    grads = mC.rasterize_voxels_backward(R, ns, W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, bg,
                                         c1.octpath, c1.centers, c1.lengths, c1.geos, rgbs, geom, binning, img, T,
                                         t(up["dC"]), t(up["dD"]) if depth else e, t(up["dN"]) if normal else e,
                                         t(up["dT"]), lR, t(up["gt"]) if lR > 0 else e, lA, lD, depth, normal, odepth,
                                         onormal)
    for mine, name in zip(grads, ("dL_dgeos", "dL_drgbs", "subdiv")):
        rel = _rel(mine.cpu().numpy(), g[name])
        assert rel < 1e-5, f"{name}: relative error {rel:.2e}"
