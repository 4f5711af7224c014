"""Full-size GPU checks on the benchmark configurations, through properties
that do not depend on the size (the oracle is too slow at these sizes):

* c4 (8M voxels, 8 views of 1920x1080, bf16 storage): the binning partitions
  the instances into per-tile ranges, every tile list is strictly increasing
  in Morton rank and holds only instances whose bbox touches the tile; the
  counting sort and the radix grouping produce the same instance array;
  images and T are bit-identical between 8x8 and 16x16 tiles and between the
  tight and the rounded pixel bbox; the backward is
  linear in the upstream gradient; no device error flag is raised.
* c3 (2M voxels, 16 uneven views): every view of the batched path (exact
  arithmetic) is bit-identical to the plain per-view path (fp32 storage).
"""
import numpy as np
import pytest
import torch

from refutil import SceneTensors, rel_err
from sv_raster_b200 import _C as mC
from sv_raster_b200 import synthetic
from sv_raster_b200.batched import BatchedRasterizer

pytestmark = pytest.mark.gpu


class DevCam:
    def __init__(self, c):
        self.width, self.height = c.width, c.height
        self.tanfovx, self.tanfovy, self.cx, self.cy, self.near = c.tanfovx, c.tanfovy, c.cx, c.cy, c.near
        self.w2c = torch.from_numpy(c.w2c).cuda()
        self.c2w = torch.from_numpy(c.c2w).cuda()


def _scene(name):
    """The seeded scene of a configuration (shared cache with bench.py)."""
    return synthetic.cached_config_scene(name)


def _octant_repeat(q):
    v = 0
    for _ in range(16):
        v = (v << 3) | q
    return v


@pytest.fixture(scope="module")
def c4():
    sc = _scene("c4")
    dev = torch.device("cuda")
    t = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dt)
    d = dict(sc=sc, octpath=t(sc.octpath.reshape(-1), torch.int64), centers=t(sc.centers), lengths=t(sc.lengths),
             geos=t(sc.geos).to(torch.bfloat16).contiguous(), sh0=t(sc.sh0).to(torch.bfloat16).contiguous(),
             shs=t(sc.shs).to(torch.bfloat16).contiguous(), cams=[DevCam(c) for c in sc.cameras])
    return d


def _raster(d, tile):
    r = BatchedRasterizer(d["cams"], d["octpath"], d["centers"], d["lengths"], max_level=d["sc"].max_level,
                          tile_size=tile)
    r.fit_capacity(d["sh0"], d["shs"], 3)
    r.prepare(d["sh0"], d["shs"], 3)
    return r


def test_c4_fullsize_binning_tiling_and_linearity(c4):
    r = _raster(c4, 8)
    color8, T8 = r.render(c4["geos"])
    torch.cuda.synchronize()
    total, err = r.header()
    assert err == 0 and total > 0 and total <= r.capacity
    a = r.arrays()
    rng = a["ranges"].long()
    lens = rng[:, 1] - rng[:, 0]
    assert int(lens.sum()) == total
    # ranges tile [0, total) without overlap
    nz = torch.nonzero(lens > 0).reshape(-1)
    starts, order = torch.sort(rng[nz, 0])
    ends = rng[nz, 1][order]
    assert int(starts[0]) == 0 and int(ends[-1]) == total
    assert torch.equal(starts[1:], ends[:-1])
    # every tile list is strictly increasing in Morton rank
    tile_of = torch.repeat_interleave(nz[order], lens[nz][order])
    vals = a["sorted_vals"][:total].long() & 0xFFFFFFFF
    vid, q = vals & ((1 << 29) - 1), vals >> 29
    reps = torch.tensor([_octant_repeat(k) for k in range(8)], dtype=torch.int64, device="cuda")
    rank = c4["octpath"][vid] ^ reps[q]
    same = tile_of[1:] == tile_of[:-1]
    assert bool(torch.all(rank[1:][same] > rank[:-1][same]))
    # instances belong to their tile: the voxel's bbox in that view touches the tile rect
    sizes = [(c.width, c.height) for c in c4["sc"].cameras]
    gx = [(w + 7) // 8 for w, h in sizes]
    gy = [(h + 7) // 8 for w, h in sizes]
    base = np.cumsum([0] + [x * y for x, y in zip(gx, gy)])
    sel = torch.randint(0, total, (200000,), device="cuda", generator=torch.Generator(device="cuda").manual_seed(3))
    ts = tile_of[sel]
    view = torch.bucketize(ts, torch.tensor(base[1:], device="cuda"), right=True)
    local = ts - torch.tensor(base, device="cuda")[view]
    gxv = torch.tensor(gx, device="cuda")[view]
    tx, ty = local % gxv, local // gxv
    bb = a["bbox"][view, vid[sel]].long() & 0xFFFFFFFF
    xmin, ymin, xmax, ymax = bb[:, 0] >> 16, bb[:, 0] & 0xFFFF, bb[:, 1] >> 16, bb[:, 1] & 0xFFFF
    gyv = torch.tensor(gy, device="cuda")[view]
    assert bool(torch.all((torch.clamp(xmin >> 3, max=gxv - 1) <= tx) & (tx <= torch.clamp(xmax >> 3, max=gxv - 1))))
    assert bool(torch.all((torch.clamp(ymin >> 3, max=gyv - 1) <= ty) & (ty <= torch.clamp(ymax >> 3, max=gyv - 1))))
    # backward is linear in the upstream gradient
    g = torch.Generator(device="cuda").manual_seed(9)
    dC = torch.randn(color8.shape, device="cuda", generator=g) * 1e-3
    dT = torch.zeros_like(T8)
    g1 = [x.clone() for x in r.backward(c4["geos"], T8, dC, dT, 3, 16)]
    g2 = [x.clone() for x in r.backward(c4["geos"], T8, 2 * dC, dT, 3, 16)]
    for x1, x2 in zip(g1, g2):
        assert rel_err(x2, 2 * x1) < 1e-5
    assert float(g1[0].abs().sum()) > 0
    # the counting sort by tile (default) and the radix passes over the tile
    # bits give the same ranges and the same sorted instance array
    assert r.binning == 1
    vals1, rng1 = a["sorted_vals"][:total].clone(), a["ranges"].clone()
    r.set_binning(0)
    r.prepare(c4["sh0"], c4["shs"], 3)
    torch.cuda.synchronize()
    assert r.header() == (total, 0)
    a0 = r.arrays()
    assert torch.equal(a0["ranges"], rng1)
    assert torch.equal(a0["sorted_vals"][:total], vals1)
    del r
    torch.cuda.empty_cache()
    # the same images with 16x16 tiles
    r16 = _raster(c4, 16)
    color16, T16 = r16.render(c4["geos"])
    torch.cuda.synchronize()
    assert r16.header()[1] == 0
    assert torch.equal(color16, color8)
    assert torch.equal(T16, T8)
    # the reference's rounded pixel bbox: more instances, the same images
    r16.set_culling(0)
    r16.fit_capacity(c4["sh0"], c4["shs"], 3)
    r16.prepare(c4["sh0"], c4["shs"], 3)
    color16r, T16r = r16.render(c4["geos"])
    torch.cuda.synchronize()
    total16r, err = r16.header()
    assert err == 0
    assert torch.equal(color16r, color8)
    assert torch.equal(T16r, T8)


def test_c3_fullsize_batched_views_equal_plain():
    sc = _scene("c3")
    C = SceneTensors(sc)
    cams = [DevCam(c) for c in sc.cameras]
    r = BatchedRasterizer(cams, C.octpath, C.centers, C.lengths, max_level=sc.max_level, tile_size=8, exact=True)
    r.fit_capacity(C.sh0, C.shs, 3)
    r.prepare(C.sh0, C.shs, 3)
    color, T = r.render(C.geos)
    torch.cuda.synchronize()
    assert r.header()[1] == 0
    cols, Ts = r.split_color(color), r.split_pixels(T)
    for k in range(len(cams)):
        cam, w2c, c2w = C.cam(k)
        ndup, geom = mC.rasterize_preprocess(cam.width, cam.height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c,
                                             c2w, cam.near, C.octpath, C.centers, C.lengths)
        vis = torch.where(ndup > 0)[0]
        rgbs = mC.sh_compute(3, vis, C.centers, c2w[:3, 3].contiguous(), C.sh0, C.shs)
        out = mC.rasterize_voxels(1, cam.width, cam.height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, 0.0,
                                  False, False, False, False, C.octpath, C.centers, C.lengths, C.geos, rgbs, geom)
        assert torch.equal(cols[k], out[3]), f"view {k}: colour differs"
        assert torch.equal(Ts[k], out[6]), f"view {k}: T differs"
