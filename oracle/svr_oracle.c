/*
 * CPU restatement of the SVRaster rasterizer hot path -- TEST INFRASTRUCTURE.
 *
 * This file is the oracle: it is used only by tests/, by
 * __graft_entry__.smoke() as the checker, and by bench.py's CPU-baseline
 * leg.  It is never part of the product path.
 *
 * It restates, one pixel at a time and without any batching, the algorithm of
 * the reference CUDA backend (panicPaul/sv_raster, backends/cuda/src):
 *   orc_preprocess     preprocessCUDA          preprocess.cu:24-132
 *   orc_binning        duplicateWithKeys +     forward.cu:518-571
 *                      stable key sort +       forward.cu:678-686
 *                      identifyTileRanges      forward.cu:576-598
 *   orc_render_fwd     FORWARD::renderCUDA     forward.cu:39-392
 *   orc_render_bwd     BACKWARD::renderCUDA    backward.cu:35-530
 *   orc_sh_fwd/_bwd    computeColorFromSH(_bw) sh_compute.cu:54-176
 *   orc_adam           (un)biased_adam_step    adam_step.cu:21-102
 * with helpers from auxiliary.h:16-321 and config.h:14-28.
 *
 * Built twice from this one source (see oracle/Makefile):
 *   REAL=float  : "mimic" mode -- fp32 with an explicit fused multiply-add
 *                 (MAD) wherever nvcc contracts a product into an add, so it
 *                 tracks the GPU to a few ulp;
 *   REAL=double : the FP64 accuracy oracle.
 * Inputs are always fp32 arrays; outputs are REAL arrays.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef REAL
#define REAL float
#endif

#ifdef ORC_DOUBLE
#define MAD(a, b, c) ((a) * (b) + (c))
#define EXP(x) exp(x)
#define SQRT(x) sqrt(x)
#define RSQRT(x) (1.0 / sqrt(x))
#define SFX(name) name##_f64
#else
#define MAD(a, b, c) fmaf((a), (b), (c))
#define EXP(x) expf(x)
#define SQRT(x) sqrtf(x)
#define RSQRT(x) (1.0f / sqrtf(x))
#define SFX(name) name##_f32
#endif

#define TILE 16
#define MAX_LEVELS 16
#define RANK_BITS 48
static const REAL MAX_ALPHA = (REAL)0.99999f;
static const REAL MIN_ALPHA = (REAL)0.00001f;
static const REAL EARLY_STOP_T = (REAL)0.0001f;
static const REAL STEP_SCALE = (REAL)100.f;

static inline REAL rmin(REAL a, REAL b) { return a < b ? a : b; }
static inline REAL rmax(REAL a, REAL b) { return a > b ? a : b; }

/* exp_linear_11 and its derivative (auxiliary.h:278-286). */
static inline REAL act(REAL x) {
  return (x > (REAL)1.1f) ? x : EXP(MAD((REAL)0.909090909091f, x, (REAL)-0.904689820196f));
}
static inline REAL act_grad(REAL x) {
  return (x > (REAL)1.1f) ? (REAL)1 : (REAL)0.909090909091f * EXP(MAD((REAL)0.909090909091f, x, (REAL)-0.904689820196f));
}
static inline REAL contract_depth(REAL x) { return (x < 1) ? x : 2 - 1 / x; }

static inline void tri_w(REAL qx, REAL qy, REAL qz, REAL w[8]) {
  const REAL x0 = 1 - qx, y0 = 1 - qy, z0 = 1 - qz;
  w[0] = x0 * y0 * z0; w[1] = x0 * y0 * qz; w[2] = x0 * qy * z0; w[3] = x0 * qy * qz;
  w[4] = qx * y0 * z0; w[5] = qx * y0 * qz; w[6] = qx * qy * z0; w[7] = qx * qy * qz;
}

typedef struct {
  REAL ox, oy, oz, dx, dy, dz, ix, iy, iz, rd_norm_inv;
  uint32_t quad;
} Ray;

static Ray make_ray(int px, int py, int W, int H, REAL tfx, REAL tfy, REAL cx, REAL cy, const float* c2w) {
  Ray r;
  const REAL cdx = ((REAL)px + (REAL)0.5f - cx) * 2 * tfx / (REAL)W;
  const REAL cdy = ((REAL)py + (REAL)0.5f - cy) * 2 * tfy / (REAL)H;
  const REAL nrm = SQRT(MAD(cdy, cdy, cdx * cdx) + 1);
  const REAL rx = MAD((REAL)c2w[1], cdy, (REAL)c2w[0] * cdx) + (REAL)c2w[2];
  const REAL ry = MAD((REAL)c2w[5], cdy, (REAL)c2w[4] * cdx) + (REAL)c2w[6];
  const REAL rz = MAD((REAL)c2w[9], cdy, (REAL)c2w[8] * cdx) + (REAL)c2w[10];
  r.rd_norm_inv = 1 / nrm;
  r.ox = c2w[3]; r.oy = c2w[7]; r.oz = c2w[11];
  r.dx = rx * r.rd_norm_inv; r.dy = ry * r.rd_norm_inv; r.dz = rz * r.rd_norm_inv;
  r.ix = 1 / r.dx; r.iy = 1 / r.dy; r.iz = 1 / r.dz;
  r.quad = ((uint32_t)(r.dx < 0) << 2) | ((uint32_t)(r.dy < 0) << 1) | (uint32_t)(r.dz < 0);
  return r;
}

static inline void ray_box(REAL cx, REAL cy, REAL cz, REAL len, const Ray* r, REAL* a, REAL* b) {
  const REAL rad = (REAL)0.5f * len;
  const REAL dx = cx - r->ox, dy = cy - r->oy, dz = cz - r->oz;
  const REAL ax = (dx - rad) * r->ix, ay = (dy - rad) * r->iy, az = (dz - rad) * r->iz;
  const REAL bx = (dx + rad) * r->ix, by = (dy + rad) * r->iy, bz = (dz + rad) * r->iz;
  *a = rmax(rmax(rmin(ax, bx), rmin(ay, by)), rmin(az, bz));
  *b = rmin(rmin(rmax(ax, bx), rmax(ay, by)), rmax(az, bz));
}

/* ------------------------------------------------------------------------- */
void SFX(orc_preprocess)(int P, int W, int H, float tanfovx, float tanfovy, float cx, float cy, const float* w2c,
                         const float* c2w, float near_plane, const float* centers, const float* lengths,
                         uint32_t* ndup, uint32_t* bbox, uint32_t* quad) {
  const int gx = (W + TILE - 1) / TILE, gy = (H + TILE - 1) / TILE;
  const float fx = 0.5f * W / tanfovx, fy = 0.5f * H / tanfovy;
  const float rox = c2w[3], roy = c2w[7], roz = c2w[11];
  for (int i = 0; i < P; ++i) {
    ndup[i] = 0; bbox[2 * i] = bbox[2 * i + 1] = 0; quad[i] = 0;
    const float vx = centers[3 * i], vy = centers[3 * i + 1], vz = centers[3 * i + 2];
    const float vr = 0.5f * lengths[i];
    const float rx = vx - rox, ry = vy - roy, rz = vz - roz;
    if (fmaf(rz, rz, fmaf(ry, ry, rx * rx)) < near_plane * near_plane) continue;
    float umin = 1e9f, vmin = 1e9f, umax = -1e9f, vmax = -1e9f;
    uint32_t qb = 0;
    for (int c = 0; c < 8; ++c) {
      const float sx = (float)(((c & 4) >> 2) * 2 - 1), sy = (float)(((c & 2) >> 1) * 2 - 1),
                  sz = (float)((c & 1) * 2 - 1);
      const float wx = fmaf(vr, sx, vx), wy = fmaf(vr, sy, vy), wz = fmaf(vr, sz, vz);
      const float camx = fmaf(w2c[2], wz, fmaf(w2c[1], wy, w2c[0] * wx)) + w2c[3];
      const float camy = fmaf(w2c[6], wz, fmaf(w2c[5], wy, w2c[4] * wx)) + w2c[7];
      const float camz = fmaf(w2c[10], wz, fmaf(w2c[9], wy, w2c[8] * wx)) + w2c[11];
      if (camz < near_plane) continue;
      const float iz = 1.0f / camz;
      const float u = camx * iz, v = camy * iz;
      const uint32_t q = ((uint32_t)(wx < rox) << 2) | ((uint32_t)(wy < roy) << 1) | (uint32_t)(wz < roz);
      umin = fminf(umin, u); vmin = fminf(vmin, v); umax = fmaxf(umax, u); vmax = fmaxf(vmax, v);
      qb |= 1u << q;
    }
    const float cxh = cx - 0.5f, cyh = cy - 0.5f;
    const float bx0 = fmaxf(fmaf(fx, umin, cxh), 0.f), by0 = fmaxf(fmaf(fy, vmin, cyh), 0.f);
    const float bx1 = fminf(fmaf(fx, umax, cxh), (float)W), by1 = fminf(fmaf(fy, vmax, cyh), (float)H);
    if (bx0 > bx1 || by0 > by1) continue;
    const uint32_t xmin = (uint32_t)lrintf(bx0), ymin = (uint32_t)lrintf(by0);
    const uint32_t xmax = (uint32_t)lrintf(bx1), ymax = (uint32_t)lrintf(by1);
    bbox[2 * i] = (xmin << 16) | ymin;
    bbox[2 * i + 1] = (xmax << 16) | ymax;
    int tx0 = (int)(xmin / TILE), ty0 = (int)(ymin / TILE), tx1 = (int)(xmax / TILE), ty1 = (int)(ymax / TILE);
    tx0 = tx0 < gx - 1 ? tx0 : gx - 1; ty0 = ty0 < gy - 1 ? ty0 : gy - 1;
    tx1 = tx1 < gx - 1 ? tx1 : gx - 1; ty1 = ty1 < gy - 1 ? ty1 : gy - 1;
    ndup[i] = (uint32_t)((1 + ty1 - ty0) * (1 + tx1 - tx0)) * (uint32_t)__builtin_popcount(qb);
    quad[i] = qb;
  }
}

/* ------------------------------------------------------------------------- */
#ifndef ORC_DOUBLE
static const uint64_t* g_keys;
static int cmp_idx(const void* a, const void* b) {
  const uint32_t ia = *(const uint32_t*)a, ib = *(const uint32_t*)b;
  if (g_keys[ia] < g_keys[ib]) return -1;
  if (g_keys[ia] > g_keys[ib]) return 1;
  return (ia > ib) - (ia < ib); /* stable: generation order breaks ties */
}

static uint64_t rep3(uint32_t q) {
  uint64_t v = 0;
  for (int l = 0; l < MAX_LEVELS; ++l) v = (v << 3) | q;
  return v;
}

/* Emits keys [tile | octpath ^ rep3(q)] and values [q<<29 | voxel] in voxel,
 * quadrant, row-major tile order, sorts them stably by key and fills the
 * per-tile [start, end) ranges.  Returns the instance count. */
int64_t orc_binning(int P, int W, int H, const int64_t* octpaths, const uint32_t* ndup, const uint32_t* bbox,
                    const uint32_t* quad, uint64_t* keys_out, uint32_t* vals_out, uint32_t* ranges) {
  const int gx = (W + TILE - 1) / TILE, gy = (H + TILE - 1) / TILE;
  int64_t n = 0;
  for (int i = 0; i < P; ++i) n += ndup[i];
  uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (n ? n : 1));
  uint32_t* vals = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  uint32_t* idx = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  int64_t off = 0;
  for (int i = 0; i < P; ++i) {
    if (!ndup[i]) continue;
    const uint32_t xmin = bbox[2 * i] >> 16, ymin = bbox[2 * i] & 0xFFFF;
    const uint32_t xmax = bbox[2 * i + 1] >> 16, ymax = bbox[2 * i + 1] & 0xFFFF;
    int tx0 = (int)(xmin / TILE), ty0 = (int)(ymin / TILE), tx1 = (int)(xmax / TILE), ty1 = (int)(ymax / TILE);
    tx0 = tx0 < gx - 1 ? tx0 : gx - 1; ty0 = ty0 < gy - 1 ? ty0 : gy - 1;
    tx1 = tx1 < gx - 1 ? tx1 : gx - 1; ty1 = ty1 < gy - 1 ? ty1 : gy - 1;
    for (uint32_t q = 0; q < 8; ++q) {
      if (!(quad[i] & (1u << q))) continue;
      const uint64_t rank = (uint64_t)octpaths[i] ^ rep3(q);
      for (int y = ty0; y <= ty1; ++y)
        for (int x = tx0; x <= tx1; ++x) {
          keys[off] = ((uint64_t)(y * gx + x) << RANK_BITS) | rank;
          vals[off] = (q << 29) | (uint32_t)i;
          ++off;
        }
    }
  }
  for (int64_t k = 0; k < n; ++k) idx[k] = (uint32_t)k;
  g_keys = keys;
  qsort(idx, (size_t)n, sizeof(uint32_t), cmp_idx);
  for (int64_t k = 0; k < n; ++k) { keys_out[k] = keys[idx[k]]; vals_out[k] = vals[idx[k]]; }
  memset(ranges, 0, sizeof(uint32_t) * 2 * (size_t)gx * gy);
  for (int64_t k = 0; k < n; ++k) {
    const uint32_t t = (uint32_t)(keys_out[k] >> RANK_BITS);
    if (k == 0 || (uint32_t)(keys_out[k - 1] >> RANK_BITS) != t) ranges[2 * t] = (uint32_t)k;
    ranges[2 * t + 1] = (uint32_t)(k + 1);
  }
  free(keys); free(vals); free(idx);
  return n;
}
#endif

/* ------------------------------------------------------------------------- */
typedef struct {
  int W, H;
  float tanfovx, tanfovy, cx, cy;
  const float* c2w;
  float bg;
  int n_samp, need_depth, need_dist, need_normal, track_max_w;
} OrcView;

static inline void load_geo(const float* geos, uint32_t vid, REAL g[8]) {
  for (int k = 0; k < 8; ++k) g[k] = geos[8 * (size_t)vid + k];
}

static inline void field_normal(const REAL g[8], REAL* nx, REAL* ny, REAL* nz) {
  *nx = ((g[4] + g[5] + g[6] + g[7]) - (g[0] + g[1] + g[2] + g[3]));
  *ny = ((g[2] + g[3] + g[6] + g[7]) - (g[0] + g[1] + g[4] + g[5]));
  *nz = ((g[1] + g[3] + g[5] + g[7]) - (g[0] + g[2] + g[4] + g[6]));
}

/* Quadrature of one ray segment [a,b] through a voxel; fills per-sample
 * alphas, dI/dgeo totals and per-sample dI/dgeo when asked. */
static REAL quadrature(const Ray* r, REAL cx, REAL cy, REAL cz, REAL l, REAL a, REAL b, const REAL g[8], int ns,
                       REAL* lalpha, REAL dI[8], REAL each[3][8]) {
  REAL vol = 0, w[8];
  const REAL linv = 1 / l;
  const REAL step = (b - a) * (ns == 1 ? (REAL)1 : ns == 2 ? (REAL)0.5f : (REAL)(1.f / 3.f));
  const REAL sx = step * r->dx, sy = step * r->dy, sz = step * r->dz;
  const REAL t0 = MAD((REAL)0.5f, step, a);
  REAL qx = (MAD(t0, r->dx, r->ox) - (cx - (REAL)0.5f * l)) * linv;
  REAL qy = (MAD(t0, r->dy, r->oy) - (cy - (REAL)0.5f * l)) * linv;
  REAL qz = (MAD(t0, r->dz, r->oz) - (cz - (REAL)0.5f * l)) * linv;
  const REAL qsx = sx * linv, qsy = sy * linv, qsz = sz * linv;
  if (dI) for (int c = 0; c < 8; ++c) dI[c] = 0;
  for (int k = 0; k < ns; ++k) {
    tri_w(qx, qy, qz, w);
    REAL d = g[0] * w[0];
    for (int c = 1; c < 8; ++c) d = MAD(g[c], w[c], d);
    const REAL a_ = act(d);
    const REAL lvi = STEP_SCALE * step * a_;
    vol = MAD(STEP_SCALE * step, a_, vol); /* nvcc fuses the sum into the product */
    if (lalpha) lalpha[k] = rmin(MAX_ALPHA, 1 - EXP(-lvi));
    if (dI) {
      const REAL dd = STEP_SCALE * step * act_grad(d);
      for (int c = 0; c < 8; ++c) {
        const REAL tmp = dd * w[c];
        dI[c] += tmp;
        if (each) each[k][c] = tmp;
      }
    }
    qx = qx + qsx; qy = qy + qsy; qz = qz + qsz;
  }
  return vol;
}

static inline int pix_in_bbox(uint32_t px, uint32_t py, const uint32_t* bb) {
  return px >= (bb[0] >> 16) && py >= (bb[0] & 0xFFFF) && px <= (bb[1] >> 16) && py <= (bb[1] & 0xFFFF);
}

/* Forward compositing of tiles [t0, t1). Outputs as the reference: color /
 * depth / normal planar [3,H,W], T [H,W], n_contrib [H,W], tile_last [T]. */
void SFX(orc_render_fwd)(const OrcView* v, int t0, int t1, const uint32_t* ranges, const uint32_t* vals,
                         const uint32_t* bbox, const float* centers, const float* lengths, const float* geos,
                         const float* rgbs, uint32_t* tile_last, uint32_t* n_contrib, REAL* color, REAL* depth,
                         REAL* normal, REAL* Tout, REAL* max_w) {
  const int W = v->W, H = v->H, gx = (W + TILE - 1) / TILE;
  const size_t HW = (size_t)W * H;
#pragma omp parallel for schedule(dynamic, 1)
  for (int t = t0; t < t1; ++t) {
    const int tx = t % gx, ty = t / gx;
    const uint32_t rb = ranges[2 * t], re = ranges[2 * t + 1];
    uint32_t tmax = 0;
    for (int ly = 0; ly < TILE; ++ly)
      for (int lx = 0; lx < TILE; ++lx) {
        const int px = tx * TILE + lx, py = ty * TILE + ly;
        if (px >= W || py >= H) continue;
        const Ray r = make_ray(px, py, W, H, v->tanfovx, v->tanfovy, v->cx, v->cy, v->c2w);
        REAL T = 1, C[3] = {0, 0, 0}, N[3] = {0, 0, 0}, D = 0, Dd = 0;
        int dmed = -1;
        REAL dmed_T = 0;
        uint32_t last = 0;
        for (uint32_t k = rb; k < re; ++k) {
          const uint32_t val = vals[k], vid = val & 0x1FFFFFFFu, q = val >> 29;
          if (!pix_in_bbox((uint32_t)px, (uint32_t)py, bbox + 2 * (size_t)vid) || q != r.quad) continue;
          const REAL cx = centers[3 * vid], cy = centers[3 * vid + 1], cz = centers[3 * vid + 2], l = lengths[vid];
          REAL a, b;
          ray_box(cx, cy, cz, l, &r, &a, &b);
          if (a > b) continue;
          REAL g[8], la[3];
          load_geo(geos, vid, g);
          const REAL vol = quadrature(&r, cx, cy, cz, l, a, b, g, v->n_samp, la, NULL, NULL);
          const REAL alpha = rmin(MAX_ALPHA, 1 - EXP(-vol));
          if (alpha < MIN_ALPHA) continue;
          const REAL pw = T * alpha;
          for (int c = 0; c < 3; ++c) C[c] = MAD(pw, (REAL)rgbs[3 * vid + c], C[c]);
          if (v->need_depth) {
            REAL dval;
            if (v->n_samp == 3) {
              const REAL ss = (REAL)0.3333333f * (b - a);
              const REAL a0 = la[0], a1 = la[1], a2 = la[2];
              const REAL q0 = a + (REAL)0.5f * ss, q1 = a + (REAL)1.5f * ss, q2 = a + (REAL)2.5f * ss;
              dval = a0 * q0 + (1 - a0) * a1 * q1 + (1 - a0) * (1 - a1) * a2 * q2;
            } else if (v->n_samp == 2) {
              const REAL ss = (REAL)0.5f * (b - a);
              const REAL a0 = la[0], a1 = la[1];
              const REAL q0 = a + (REAL)0.5f * ss, q1 = a + (REAL)1.5f * ss;
              dval = a0 * q0 + (1 - a0) * a1 * q1;
            } else {
              dval = alpha * (REAL)0.5f * (a + b);
            }
            D = MAD(T, dval, D);
            if (T > (REAL)0.5f) { dmed = (int)vid; dmed_T = T; }
          }
          if (v->need_dist) Dd = MAD(pw * (REAL)0.5f, contract_depth(a) + contract_depth(b), Dd);
          if (v->need_normal) {
            REAL nx, ny, nz;
            field_normal(g, &nx, &ny, &nz);
            const REAL rl = 1 / SQRT(nx * nx + ny * ny + nz * nz + (REAL)1e-15f);
            N[0] = MAD(pw * rl, nx, N[0]); N[1] = MAD(pw * rl, ny, N[1]); N[2] = MAD(pw * rl, nz, N[2]);
          }
          T *= (1 - alpha);
          last = k - rb + 1;
          if (v->track_max_w && max_w && pw > max_w[vid]) {
#pragma omp critical
            { if (pw > max_w[vid]) max_w[vid] = pw; }
          }
          if (T < EARLY_STOP_T) break;
        }
        REAL Dmed = 0;
        if (v->need_depth && dmed != -1) {
          const REAL cx = centers[3 * dmed], cy = centers[3 * dmed + 1], cz = centers[3 * dmed + 2], l = lengths[dmed];
          REAL a, b, g[8], w[8];
          ray_box(cx, cy, cz, l, &r, &a, &b);
          load_geo(geos, (uint32_t)dmed, g);
          const REAL linv = 1 / l, step = (b - a) * (REAL)0.0625f;
          const REAL t0_ = MAD((REAL)0.5f, step, a);
          REAL qx = (MAD(t0_, r.dx, r.ox) - (cx - (REAL)0.5f * l)) * linv;
          REAL qy = (MAD(t0_, r.dy, r.oy) - (cy - (REAL)0.5f * l)) * linv;
          REAL qz = (MAD(t0_, r.dz, r.oz) - (cz - (REAL)0.5f * l)) * linv;
          const REAL qsx = step * r.dx * linv, qsy = step * r.dy * linv, qsz = step * r.dz * linv;
          Dmed = a - (REAL)0.5f * step;
          for (int k = 0; k < 16 && dmed_T > (REAL)0.5f; ++k) {
            Dmed += step;
            tri_w(qx, qy, qz, w);
            REAL d = g[0] * w[0];
            for (int c = 1; c < 8; ++c) d = MAD(g[c], w[c], d);
            dmed_T *= EXP(-(STEP_SCALE * step * act(d)));
            qx += qsx; qy += qsy; qz += qsz;
          }
        }
        const size_t pid = (size_t)py * W + px;
        n_contrib[pid] = last;
        if (last > tmax) tmax = last;
        for (int c = 0; c < 3; ++c) color[c * HW + pid] = MAD(T, (REAL)v->bg, C[c]);
        Tout[pid] = T;
        if (v->need_depth && depth) { depth[pid] = D * r.rd_norm_inv; depth[2 * HW + pid] = Dmed * r.rd_norm_inv; }
        if (v->need_dist && depth) depth[HW + pid] = Dd;
        if (v->need_normal && normal) for (int c = 0; c < 3; ++c) normal[c * HW + pid] = N[c];
      }
    tile_last[t] = rb + tmax;
  }
}

/* Backward of tiles [t0, t1): accumulates dL_dgeos [P,8], dL_drgbs [P,3],
 * subdiv [P] (REAL, caller-zeroed).  Mirrors backward.cu:35-530. */
void SFX(orc_render_bwd)(const OrcView* v, int t0, int t1, const uint32_t* ranges, const uint32_t* tile_last,
                         const uint32_t* vals, const uint32_t* bbox, const float* centers, const float* lengths,
                         const float* geos, const float* rgbs, const uint32_t* n_contrib, const REAL* Tfinal,
                         const float* dL_dcolor, const float* dL_ddepth, const float* dL_dnormal, const float* dL_dT,
                         float lambda_R, const float* gt, float lambda_asc, float lambda_dist, const REAL* out_depth,
                         REAL* dL_dgeos, REAL* dL_drgbs, REAL* subdiv) {
  const int W = v->W, H = v->H, gx = (W + TILE - 1) / TILE;
  const size_t HW = (size_t)W * H;
  const REAL WHinv = 1 / ((REAL)(W * H));
  const REAL wR = lambda_R * WHinv, wA = lambda_asc * WHinv, wD = lambda_dist * WHinv;
#pragma omp parallel for schedule(dynamic, 1)
  for (int t = t0; t < t1; ++t) {
    const int tx = t % gx, ty = t / gx;
    const uint32_t rb = ranges[2 * t];
    (void)tile_last;
    for (int ly = 0; ly < TILE; ++ly)
      for (int lx = 0; lx < TILE; ++lx) {
        const int px = tx * TILE + lx, py = ty * TILE + ly;
        if (px >= W || py >= H) continue;
        const size_t pid = (size_t)py * W + px;
        const Ray r = make_ray(px, py, W, H, v->tanfovx, v->tanfovy, v->cx, v->cy, v->c2w);
        REAL T = Tfinal[pid];
        const REAL g3[3] = {dL_dcolor[pid], dL_dcolor[HW + pid], dL_dcolor[2 * HW + pid]};
        REAL last_dT = MAD((REAL)v->bg, g3[0] + g3[1] + g3[2], (REAL)dL_dT[pid]);
        const REAL dD = v->need_depth ? (REAL)dL_ddepth[pid] * r.rd_norm_inv : 0;
        REAL dN[3] = {0, 0, 0};
        if (v->need_normal) for (int c = 0; c < 3; ++c) dN[c] = dL_dnormal[c * HW + pid];
        REAL gtp[3] = {0, 0, 0};
        if (lambda_R > 0) for (int c = 0; c < 3; ++c) gtp[c] = gt[c * HW + pid];
        REAL pre_wm = 0, suf_wm = 0, pre_w = 0, suf_w = 0;
        if (v->need_dist) { pre_wm = out_depth[HW + pid]; pre_w = 1 - Tfinal[pid]; }
        const uint32_t nc = n_contrib[pid];
        for (int64_t pos = (int64_t)nc - 1; pos >= 0; --pos) {
          const uint32_t k = rb + (uint32_t)pos;
          const uint32_t val = vals[k], vid = val & 0x1FFFFFFFu, q = val >> 29;
          if (!pix_in_bbox((uint32_t)px, (uint32_t)py, bbox + 2 * (size_t)vid) || q != r.quad) continue;
          const REAL cx = centers[3 * vid], cy = centers[3 * vid + 1], cz = centers[3 * vid + 2], l = lengths[vid];
          REAL a, b;
          ray_box(cx, cy, cz, l, &r, &a, &b);
          if (a > b) continue;
          REAL g[8], dI[8], each[3][8], la[3], dg[8] = {0, 0, 0, 0, 0, 0, 0, 0};
          load_geo(geos, vid, g);
          const REAL vol = quadrature(&r, cx, cy, cz, l, a, b, g, v->n_samp, la, dI, each);
          const REAL eneg = EXP(-vol);
          const REAL alpha = rmin(MAX_ALPHA, 1 - eneg);
          if (alpha < MIN_ALPHA) continue;
          T = T / (1 - alpha);
          const REAL pw = alpha * T;
          const REAL c3[3] = {rgbs[3 * vid], rgbs[3 * vid + 1], rgbs[3 * vid + 2]};
          REAL dpw = MAD(g3[2], c3[2], MAD(g3[1], c3[1], g3[0] * c3[0]));
          if (v->need_dist) {
            const REAL ad = contract_depth(a), bd = contract_depth(b);
            const REAL m = (REAL)0.5f * (ad + bd), wm = m * pw;
            pre_wm -= wm; pre_w -= pw;
            const REAL uni = (REAL)0.6666666f * pw * (bd - ad);
            const REAL bi = 2 * (m * (pre_w - suf_w) - (pre_wm - suf_wm));
            dpw += wD * (uni + bi);
            suf_wm += wm; suf_w += pw;
          }
          if (v->need_normal) {
            REAL nx, ny, nz;
            field_normal(g, &nx, &ny, &nz);
            const REAL rl = 1 / SQRT(nx * nx + ny * ny + nz * nz + (REAL)1e-15f);
            const REAL sx = rl * nx, sy = rl * ny, sz = rl * nz;
            dpw += dN[0] * sx + dN[1] * sy + dN[2] * sz;
            const REAL dsx = pw * dN[0], dsy = pw * dN[1], dsz = pw * dN[2];
            const REAL dt = dsx * nx + dsy * ny + dsz * nz;
            const REAL lx_ = rl * (dsx - dt * rl * sx), ly_ = rl * (dsy - dt * rl * sy), lz_ = rl * (dsz - dt * rl * sz);
            dg[0] += -lx_ - ly_ - lz_; dg[1] += -lx_ - ly_ + lz_; dg[2] += -lx_ + ly_ - lz_; dg[3] += -lx_ + ly_ + lz_;
            dg[4] += +lx_ - ly_ - lz_; dg[5] += +lx_ - ly_ + lz_; dg[6] += +lx_ + ly_ - lz_; dg[7] += +lx_ + ly_ + lz_;
          }
          const REAL dalpha = T * (dpw - last_dT);
          last_dT = MAD(alpha, dpw - last_dT, last_dT);
          const REAL dIv = dalpha * eneg;
          for (int c = 0; c < 8; ++c) dg[c] = MAD(dIv, dI[c], dg[c]);
          if (v->need_depth) {
            REAL dval, dLI[3];
            if (v->n_samp == 3) {
              const REAL ss = (REAL)0.3333333f * (b - a);
              const REAL a0 = la[0], a1 = la[1], a2 = la[2];
              const REAL q0 = a + (REAL)0.5f * ss, q1 = a + (REAL)1.5f * ss, q2 = a + (REAL)2.5f * ss;
              dval = a0 * q0 + (1 - a0) * a1 * q1 + (1 - a0) * (1 - a1) * a2 * q2;
              dLI[0] = dD * T * (q0 + a1 * a2 * q2 - a1 * q1 - a2 * q2) * (1 - a0);
              dLI[1] = dD * T * (q1 + a0 * a2 * q2 - a0 * q1 - a2 * q2) * (1 - a1);
              dLI[2] = dD * T * (q2 + a0 * a1 * q2 - a0 * q2 - a1 * q2) * (1 - a2);
              for (int c = 0; c < 8; ++c) dg[c] += dLI[0] * each[0][c] + dLI[1] * each[1][c] + dLI[2] * each[2][c];
            } else if (v->n_samp == 2) {
              const REAL ss = (REAL)0.5f * (b - a);
              const REAL a0 = la[0], a1 = la[1];
              const REAL q0 = a + (REAL)0.5f * ss, q1 = a + (REAL)1.5f * ss;
              dval = a0 * q0 + (1 - a0) * a1 * q1;
              dLI[0] = dD * T * (q0 - a1 * q1) * (1 - a0);
              dLI[1] = dD * T * (q1 - a0 * q1) * (1 - a1);
              for (int c = 0; c < 8; ++c) dg[c] += dLI[0] * each[0][c] + dLI[1] * each[1][c];
            } else {
              const REAL q0 = (REAL)0.5f * (a + b);
              dval = alpha * q0;
              dLI[0] = dD * T * q0 * (1 - alpha);
              for (int c = 0; c < 8; ++c) dg[c] += dLI[0] * dI[c];
            }
            last_dT += dD * dval;
          }
          if (lambda_asc > 0) {
            const REAL linv = 1 / l;
            const REAL lox = cx - (REAL)0.5f * l, loy = cy - (REAL)0.5f * l, loz = cz - (REAL)0.5f * l;
            REAL wa[8], wb[8];
            tri_w((MAD(a, r.dx, r.ox) - lox) * linv, (MAD(a, r.dy, r.oy) - loy) * linv,
                  (MAD(a, r.dz, r.oz) - loz) * linv, wa);
            tri_w((MAD(b, r.dx, r.ox) - lox) * linv, (MAD(b, r.dy, r.oy) - loy) * linv,
                  (MAD(b, r.dz, r.oz) - loz) * linv, wb);
            REAL da = 0, db = 0;
            for (int c = 0; c < 8; ++c) { da += g[c] * wa[c]; db += g[c] * wb[c]; }
            const REAL rw = wA * pw * (REAL)(da > db);
            for (int c = 0; c < 8; ++c) dg[c] += rw * (wa[c] - wb[c]);
          }
          REAL dr[3];
          for (int c = 0; c < 3; ++c) {
            dr[c] = pw * g3[c];
            if (lambda_R > 0) dr[c] += wR * pw * 2 * (c3[c] - gtp[c]);
          }
          const REAL sub = fabs((double)(dalpha * alpha));
          for (int c = 0; c < 8; ++c) {
#pragma omp atomic
            dL_dgeos[8 * (size_t)vid + c] += dg[c];
          }
          for (int c = 0; c < 3; ++c) {
#pragma omp atomic
            dL_drgbs[3 * (size_t)vid + c] += dr[c];
          }
#pragma omp atomic
          subdiv[vid] += sub;
        }
      }
  }
}

/* ------------------------------------------------------------------------- */
static const double SH_C0 = 0.28209479177387814, SH_C1 = 0.4886025119029199;
static const double SH_C2[5] = {1.0925484305920792, -1.0925484305920792, 0.31539156525252005, -1.0925484305920792,
                                0.5462742152960396};
static const double SH_C3[7] = {-0.5900435899266435, 2.890611442640554, -0.4570457994644658, 0.3731763325901154,
                                -0.4570457994644658, 1.445305721320277, -0.5900435899266435};

static void sh_basis(REAL x, REAL y, REAL z, REAL bs[16]) {
  const REAL xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
  bs[0] = (REAL)SH_C0;
  bs[1] = -(REAL)SH_C1 * y; bs[2] = (REAL)SH_C1 * z; bs[3] = -(REAL)SH_C1 * x;
  bs[4] = (REAL)SH_C2[0] * xy; bs[5] = (REAL)SH_C2[1] * yz; bs[6] = (REAL)SH_C2[2] * (2 * zz - xx - yy);
  bs[7] = (REAL)SH_C2[3] * xz; bs[8] = (REAL)SH_C2[4] * (xx - yy);
  bs[9] = (REAL)SH_C3[0] * y * (3 * xx - yy); bs[10] = (REAL)SH_C3[1] * xy * z;
  bs[11] = (REAL)SH_C3[2] * y * (4 * zz - xx - yy); bs[12] = (REAL)SH_C3[3] * z * (2 * zz - 3 * xx - 3 * yy);
  bs[13] = (REAL)SH_C3[4] * x * (4 * zz - xx - yy); bs[14] = (REAL)SH_C3[5] * z * (xx - yy);
  bs[15] = (REAL)SH_C3[6] * x * (xx - 3 * yy);
}

/* rgb = max(sum_k basis_k(dir) * sh_k + 0.5, 0), dir = normalize(c - cam). */
void SFX(orc_sh_fwd)(int deg, int n, const int64_t* idx, int M, const float* centers, const float* campos,
                     const float* sh0, const float* shs, REAL* rgbs) {
  const int nb = (deg + 1) * (deg + 1);
  for (int t = 0; t < n; ++t) {
    const int64_t i = idx[t];
    REAL x = (REAL)centers[3 * i] - (REAL)campos[0], y = (REAL)centers[3 * i + 1] - (REAL)campos[1],
         z = (REAL)centers[3 * i + 2] - (REAL)campos[2];
    const REAL rn = 1 / SQRT(x * x + y * y + z * z);
    x *= rn; y *= rn; z *= rn;
    REAL bs[16];
    sh_basis(x, y, z, bs);
    for (int c = 0; c < 3; ++c) {
      REAL v = bs[0] * sh0[3 * i + c];
      for (int k = 1; k < nb; ++k) v += bs[k] * shs[((size_t)i * (M - 1) + (k - 1)) * 3 + c];
      v += (REAL)0.5;
      rgbs[3 * i + c] = v > 0 ? v : 0;
    }
  }
}

void SFX(orc_sh_bwd)(int deg, int n, const int64_t* idx, int M, const float* centers, const float* campos,
                     const float* dL_drgb, REAL* dsh0, REAL* dshs) {
  const int nb = (deg + 1) * (deg + 1);
  for (int t = 0; t < n; ++t) {
    const int64_t i = idx[t];
    REAL x = (REAL)centers[3 * i] - (REAL)campos[0], y = (REAL)centers[3 * i + 1] - (REAL)campos[1],
         z = (REAL)centers[3 * i + 2] - (REAL)campos[2];
    const REAL rn = 1 / SQRT(x * x + y * y + z * z);
    x *= rn; y *= rn; z *= rn;
    REAL bs[16];
    sh_basis(x, y, z, bs);
    for (int c = 0; c < 3; ++c) {
      dsh0[3 * i + c] = bs[0] * dL_drgb[3 * i + c];
      for (int k = 1; k < nb; ++k) dshs[((size_t)i * (M - 1) + (k - 1)) * 3 + c] = bs[k] * dL_drgb[3 * i + c];
    }
  }
}

/* Adam in place (adam_step.cu:21-102); bias terms in double on the host side. */
void SFX(orc_adam)(int biased, int sparse, int64_t n, REAL* p, const float* g, REAL* m, REAL* v, double step,
                   double lr, double b1, double b2, float eps) {
  const double bc1 = 1.0 - pow(b1, step), bc2 = 1.0 - pow(b2, step);
  const REAL step_size = biased ? (REAL)(float)lr : (REAL)(float)(lr / bc1);
  const REAL rbc2 = (REAL)(float)(1.0 / sqrt(bc2));
  const REAL B1 = (REAL)(float)b1, B2 = (REAL)(float)b2;
  for (int64_t i = 0; i < n; ++i) {
    const REAL gi = g[i];
    if (sparse && gi == 0) continue;
    const REAL mi = MAD(B1, m[i], MAD(-B1, gi, gi));
    const REAL vi = MAD(B2, v[i], MAD(-B2, gi * gi, gi * gi));
    const REAL den = biased ? SQRT(vi) + (REAL)eps : MAD(SQRT(vi), rbc2, (REAL)eps);
    p[i] = p[i] - step_size * (mi / den);
    m[i] = mi;
    v[i] = vi;
  }
}
