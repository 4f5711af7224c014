// C ABI implementation: buffer layouts, argument checks and launch sequences
// of the plain (one view per call) path.  See include/svr_b200.h.
#include <cmath>
#include <cstring>
#include <atomic>

#include "../../include/svr_b200.h"
#include "svr_common.cuh"
#include "svr_kernels.h"
#include "svr_render.cuh"
#include "svr_render_bwd.cuh"
#include "svr_render_fwd.cuh"

using namespace svr;

namespace {

constexpr size_t kAlign = 256;

inline size_t align_up(size_t x, size_t a = kAlign) { return (x + a - 1) / a * a; }

// Sequential carve of a caller buffer into aligned sub-arrays, relative to
// the buffer start (so sizes do not depend on the base address).
struct Carver {
  char* base;
  size_t off = 0;
  explicit Carver(void* b) : base(static_cast<char*>(b)) {}
  template <typename T>
  T* take(size_t count) {
    off = align_up(off);
    T* p = reinterpret_cast<T*>(base + off);
    off += count * sizeof(T);
    return p;
  }
  size_t size() const { return align_up(off) + kAlign; }
};

// ---- geom buffer: header | n_dup | scan | bbox | quad | scan temp -------------
struct GeomLayout {
  uint32_t* header;  // [0] instance count, [1] device error word
  uint32_t* ndup;
  uint32_t* scan;
  uint2* bbox;
  uint32_t* quad;
  void* scan_temp;
  size_t bytes;
};

GeomLayout geom_layout(void* buf, int64_t P) {
  Carver c(buf);
  GeomLayout g;
  g.header = c.take<uint32_t>(16);
  g.ndup = c.take<uint32_t>(P);
  g.scan = c.take<uint32_t>(P);
  g.bbox = c.take<uint2>(P);
  g.quad = c.take<uint32_t>(P);
  g.scan_temp = c.take<char>(scan_temp_bytes((size_t)P));
  g.bytes = c.size();
  return g;
}

// ---- image buffer: ranges | tile_last | n_contrib | tile work orders ---------
struct ImageLayout {
  uint2* ranges;
  uint32_t* tile_last;
  uint32_t* n_contrib;
  uint32_t* order;      // [T] tiles largest first (by list length), written by the
                        // render call, read by the forward and backward launches
  uint64_t* okey;       // [2T] order sort keys
  uint32_t* oval;       // [T]
  uint32_t* ocount;     // tile count read by the order sort
  void* otemp;          // tile_order_temp_bytes(T)
  size_t bytes;
};

inline int tiles_x(int W) { return (W + kTileX - 1) / kTileX; }
inline int tiles_y(int H) { return (H + kTileY - 1) / kTileY; }

ImageLayout image_layout(void* buf, int W, int H) {
  Carver c(buf);
  ImageLayout im;
  const size_t T = (size_t)tiles_x(W) * tiles_y(H);
  im.ranges = c.take<uint2>(T);
  im.tile_last = c.take<uint32_t>(T);
  im.n_contrib = c.take<uint32_t>((size_t)W * H);
  im.order = c.take<uint32_t>(T);
  im.okey = c.take<uint64_t>(2 * T);
  im.oval = c.take<uint32_t>(T);
  im.ocount = c.take<uint32_t>(1);
  im.otemp = c.take<char>(tile_order_temp_bytes((uint32_t)T));
  im.bytes = c.size();
  return im;
}

// ---- binning buffer: keys a/b | vals a/b | sort temp ---------------------------
struct BinningLayout {
  uint64_t* keys_a;
  uint64_t* keys_b;
  uint32_t* vals_a;
  uint32_t* vals_b;
  void* sort_temp;
  size_t bytes;
};

// The sort temp (last) serves the tile-bit radix passes and then the
// per-tile segment sort, so its size depends on the tile count; the stages
// after binning only use the key/value arrays and pass n_tiles = 0.
BinningLayout binning_layout(void* buf, size_t n, int n_tiles) {
  Carver c(buf);
  BinningLayout b;
  b.keys_a = c.take<uint64_t>(n);
  b.keys_b = c.take<uint64_t>(n);
  b.vals_a = c.take<uint32_t>(n);
  b.vals_b = c.take<uint32_t>(n);
  b.sort_temp = c.take<char>(std::max(sort_temp_bytes(n), n_tiles > 0 ? seg_sort_temp_bytes(n, n_tiles) : 0));
  b.bytes = c.size();
  return b;
}

// 21-level binning: the 16-level layout, then the wide keys' high halves
// and the per-instance rank, tile and value arrays.
DeepBinning deep_layout(void* buf, size_t n, int n_tiles, size_t* bytes) {
  BinningLayout bl = binning_layout(buf, n, n_tiles);
  Carver c(buf ? static_cast<char*>(buf) + bl.bytes : nullptr);
  DeepBinning d;
  d.keys_a = bl.keys_a;
  d.keys_b = bl.keys_b;
  d.vals_a = bl.vals_a;
  d.vals_b = bl.vals_b;
  d.sort_temp = bl.sort_temp;
  d.vals_out = bl.vals_b;
  d.keys_lo = bl.keys_b;
  d.keys_hi = c.take<uint64_t>(n);
  d.rank_of = c.take<uint64_t>(n);
  d.tile_of = c.take<uint32_t>(n);
  d.val_of = c.take<uint32_t>(n);
  if (bytes) *bytes = bl.bytes + c.size();
  return d;
}

// Bits needed to represent n (the tile-id width of the sort key).
inline int bit_width_u32(uint32_t n) {
  int b = 0;
  while (b < 32 && (n >> b)) ++b;
  return b;
}

inline int plain_key_bits(int W, int H) { return kRankBits + bit_width_u32((uint32_t)(tiles_x(W) * tiles_y(H))); }

ViewParams make_view(const svr_camera& cam) {
  ViewParams v;
  memset(&v, 0, sizeof(v));
  v.W = cam.width;
  v.H = cam.height;
  v.grid_x = tiles_x(cam.width);
  v.grid_y = tiles_y(cam.height);
  v.tile_shift = kTileShift;
  v.tanfovx = cam.tanfovx;
  v.tanfovy = cam.tanfovy;
  v.cx = cam.cx;
  v.cy = cam.cy;
  // Same float arithmetic as the reference host code (preprocess.cu:173-174).
  v.focal_x = 0.5f * cam.width / cam.tanfovx;
  v.focal_y = 0.5f * cam.height / cam.tanfovy;
  v.near_plane = cam.near_plane;
  v.bg = cam.bg_color;
  v.w2c = cam.w2c;
  v.c2w = cam.c2w;
  return v;
}

inline bool valid_camera(const svr_camera* cam) {
  return cam && cam->width > 0 && cam->height > 0 && cam->width < 65536 && cam->height < 65536 && cam->w2c &&
         cam->c2w;
}

inline int check_launch(int debug, cudaStream_t stream) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return SVR_ERR_CUDA;
  if (debug) {
    e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return SVR_ERR_CUDA;
  }
  return SVR_OK;
}

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

extern "C" {

int svr_max_num_levels(void) { return kMaxLevels; }
float svr_step_sz_scale(void) { return kStepScale; }
int svr_max_n_samp(void) { return kMaxSamples; }
int svr_version(void) { return 1; }

const char* svr_status_string(int s) {
  switch (s) {
    case SVR_OK: return "ok";
    case SVR_ERR_SHAPE: return "invalid sizes or arguments";
    case SVR_ERR_CAPACITY: return "buffer capacity exceeded";
    case SVR_ERR_KEYBITS: return "sort key does not fit in 64 bits";
    case SVR_ERR_CUDA: return "CUDA runtime error";
    case SVR_ERR_DEVICE: return "device-side consistency check failed";
    case SVR_ERR_ALIGN: return "pointer alignment requirement not met";
    default: return "unknown status";
  }
}

size_t svr_geom_buffer_bytes(int64_t P) { return P < 0 ? 0 : geom_layout(nullptr, P).bytes; }
size_t svr_image_buffer_bytes(int width, int height) {
  return (width <= 0 || height <= 0) ? 0 : image_layout(nullptr, width, height).bytes;
}
size_t svr_binning_buffer_bytes(int64_t n, int width, int height) {
  if (n < 0 || width <= 0 || height <= 0) return 0;
  return binning_layout(nullptr, (size_t)n, tiles_x(width) * tiles_y(height)).bytes;
}

size_t svr_binning_buffer_bytes_levels(int64_t n, int width, int height, int levels) {
  if (levels == kMaxLevels) return svr_binning_buffer_bytes(n, width, height);
  if (levels != kDeepLevels || n < 0 || width <= 0 || height <= 0) return 0;
  size_t bytes = 0;
  deep_layout(nullptr, (size_t)n, tiles_x(width) * tiles_y(height), &bytes);
  return bytes;
}

const uint32_t* svr_geom_count_ptr(const void* geom) { return static_cast<const uint32_t*>(geom); }
uint32_t* svr_geom_error_ptr(void* geom) { return static_cast<uint32_t*>(geom) + 1; }

int svr_rasterize_preprocess(const svr_camera* cam, int64_t P, const int64_t* octree_paths, const float* vox_centers,
                             const float* vox_lengths, int32_t* out_n_duplicates, void* geom_buffer,
                             size_t geom_bytes, int debug, void* stream_) {
  (void)octree_paths;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  if (P < 0 || P >= (1ll << kVoxIdBits) || !valid_camera(cam)) return SVR_ERR_SHAPE;
  if (P == 0) return SVR_OK;
  GeomLayout g = geom_layout(geom_buffer, P);
  if (!geom_buffer || geom_bytes < g.bytes || !vox_centers || !vox_lengths || !out_n_duplicates) return SVR_ERR_SHAPE;
  ViewTable vt;
  vt.n = 1;
  vt.v[0] = make_view(*cam);
  cudaMemsetAsync(g.header, 0, 16 * sizeof(uint32_t), stream);
  launch_preprocess(vt, (int)P, vox_centers, vox_lengths, out_n_duplicates, g.ndup, g.bbox, g.quad, stream);
  launch_scan_inclusive(g.ndup, g.scan, (size_t)P, g.scan_temp, g.header, 0xffffffffull, g.header + 1, stream);
  return check_launch(debug, stream);
}

// Shared argument checks and layouts of the forward stages.
struct FwdCtx {
  ViewTable vt;
  GeomLayout g;
  ImageLayout im;
  BinningLayout bl;
  size_t n;
  int key_bits;
};

static int fwd_prepare(const svr_camera* cam, int n_samp, int64_t P, int64_t num_rendered, void* geom_buffer,
                       void* binning_buffer, size_t binning_bytes, void* image_buffer, size_t image_bytes,
                       FwdCtx& c, bool deep = false) {
  if (!valid_camera(cam) || n_samp < 1 || n_samp > kMaxSamples || P < 0 || num_rendered < 0 ||
      num_rendered > 0xffffffffll)
    return SVR_ERR_SHAPE;
  const int W = cam->width, H = cam->height;
  c.im = image_layout(image_buffer, W, H);
  if (!image_buffer || image_bytes < c.im.bytes) return SVR_ERR_CAPACITY;
  c.n = (size_t)num_rendered;
  c.bl = binning_layout(binning_buffer, c.n, tiles_x(W) * tiles_y(H));
  // (21-level binning checks its own, larger buffer; its keys are two words wide)
  if (!deep && c.n > 0 && (!binning_buffer || binning_bytes < c.bl.bytes)) return SVR_ERR_CAPACITY;
  c.key_bits = plain_key_bits(W, H);
  if (!deep && c.key_bits > 64) return SVR_ERR_KEYBITS;
  c.g = geom_layout(geom_buffer, P);
  c.vt.n = 1;
  c.vt.v[0] = make_view(*cam);
  return SVR_OK;
}

int svr_rasterize_binning(const svr_camera* cam, int64_t P, int64_t num_rendered, const int64_t* octree_paths,
                          void* geom_buffer, void* binning_buffer, size_t binning_bytes, void* image_buffer,
                          size_t image_bytes, int debug, void* stream_) {
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  FwdCtx c;
  int st = fwd_prepare(cam, 1, P, num_rendered, geom_buffer, binning_buffer, binning_bytes, image_buffer,
                       image_bytes, c);
  if (st != SVR_OK) return st;
  if (P == 0) return SVR_OK;
  if (c.n > 0 && !octree_paths) return SVR_ERR_SHAPE;
  const ViewParams& vp = c.vt.v[0];
  cudaMemsetAsync(c.im.ranges, 0, (size_t)vp.grid_x * vp.grid_y * sizeof(uint2), stream);
  if (c.n > 0) {
    // Two-level sort (same order as one stable sort by the full key): radix
    // passes over the tile bits leave each tile's instances together, in
    // generation order, in (keys_a, vals_a); the per-tile segment sort by the
    // rank bits then writes the final order to (keys_b, vals_b).
    const bool odd = (sort_passes(c.key_bits - kRankBits) & 1) != 0;
    uint64_t* k0 = odd ? c.bl.keys_b : c.bl.keys_a;
    uint32_t* v0 = odd ? c.bl.vals_b : c.bl.vals_a;
    uint64_t* k1 = odd ? c.bl.keys_a : c.bl.keys_b;
    uint32_t* v1 = odd ? c.bl.vals_a : c.bl.vals_b;
    const int n_tiles = vp.grid_x * vp.grid_y;
    launch_duplicate(c.vt, (int)P, octree_paths, c.g.bbox, c.g.quad, c.g.ndup, c.g.scan, k0, v0, (uint32_t)c.n,
                     c.g.header + 1, stream);
    launch_radix_sort(k0, v0, k1, v1, nullptr, c.g.header, (uint32_t)c.n, c.key_bits, c.bl.sort_temp, stream,
                      kRankBits);
    launch_tile_ranges(c.bl.keys_a, nullptr, c.g.header, (uint32_t)c.n, kRankBits, 0u, (uint32_t)n_tiles,
                       c.im.ranges, stream);
    launch_tile_segment_sort(c.im.ranges, n_tiles, c.bl.keys_a, c.bl.vals_a, c.bl.keys_b, c.bl.vals_b, kRankBits,
                             c.n, c.bl.sort_temp, stream);
  }
  return check_launch(debug, stream);
}

int svr_rasterize_render(const svr_camera* cam, int n_samp, int need_depth, int need_distortion, int need_normal,
                         int track_max_w, int64_t P, int64_t num_rendered, const float* vox_centers,
                         const float* vox_lengths, const float* geos, const float* rgbs, void* geom_buffer,
                         void* binning_buffer, size_t binning_bytes, void* image_buffer, size_t image_bytes,
                         float* out_color, float* out_depth, float* out_normal, float* out_T, float* max_w, int debug,
                         void* stream_) {
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  FwdCtx c;
  int st = fwd_prepare(cam, n_samp, P, num_rendered, geom_buffer, binning_buffer, binning_bytes, image_buffer,
                       image_bytes, c);
  if (st != SVR_OK) return st;
  if (P == 0) return SVR_OK;
  if (!out_color || !out_T || ((need_depth || need_distortion) && !out_depth) || (need_normal && !out_normal) ||
      (track_max_w && !max_w) || !geos || !rgbs || !vox_centers || !vox_lengths)
    return SVR_ERR_SHAPE;
  if (!aligned16(geos)) return SVR_ERR_ALIGN;
  VoxelArrays va{c.g.bbox, vox_centers, vox_lengths, geos, nullptr, rgbs};
  FwdTileOut out{c.im.tile_last, c.im.n_contrib, out_color, out_depth, out_normal, out_T, max_w};
  const uint32_t n_tiles = (uint32_t)(c.vt.v[0].grid_x * c.vt.v[0].grid_y);
  cudaMemsetAsync(c.im.tile_last, 0, n_tiles * sizeof(uint32_t), stream);  // combined by atomicMax
  launch_tile_order(c.im.ranges, nullptr, n_tiles, c.im.okey, c.im.oval, c.im.order, c.im.ocount, c.im.otemp,
                    stream);
  launch_render_fwd(c.vt.v[0], c.im.ranges, c.n > 0 ? c.bl.vals_b : nullptr, va, out, n_samp, need_depth != 0,
                    need_distortion != 0, need_normal != 0, track_max_w != 0, c.im.order, stream);
  return check_launch(debug, stream);
}

int svr_rasterize_binning_levels(const svr_camera* cam, int64_t P, int64_t num_rendered, const int64_t* octree_paths,
                                 int levels, void* geom_buffer, void* binning_buffer, size_t binning_bytes,
                                 void* image_buffer, size_t image_bytes, int debug, void* stream_) {
  if (levels == kMaxLevels)
    return svr_rasterize_binning(cam, P, num_rendered, octree_paths, geom_buffer, binning_buffer, binning_bytes,
                                 image_buffer, image_bytes, debug, stream_);
  if (levels != kDeepLevels) return SVR_ERR_SHAPE;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  FwdCtx c;
  int st = fwd_prepare(cam, 1, P, num_rendered, geom_buffer, binning_buffer, 0, image_buffer, image_bytes, c, true);
  if (st != SVR_OK) return st;
  size_t need = 0;
  const ViewParams& vp = c.vt.v[0];
  const int n_tiles = vp.grid_x * vp.grid_y;
  DeepBinning d = deep_layout(binning_buffer, c.n, n_tiles, &need);
  if (c.n > 0 && (!binning_buffer || binning_bytes < need)) return SVR_ERR_CAPACITY;
  if (P == 0) return SVR_OK;
  if (c.n > 0 && !octree_paths) return SVR_ERR_SHAPE;
  cudaMemsetAsync(c.im.ranges, 0, (size_t)n_tiles * sizeof(uint2), stream);
  launch_binning_deep(vp, (int)P, octree_paths, c.g.bbox, c.g.quad, c.g.ndup, c.g.scan, c.g.header, (uint32_t)c.n, d,
                      c.im.ranges, c.g.header + 1, stream);
  return check_launch(debug, stream);
}

int svr_rasterize_forward_levels(const svr_camera* cam, int n_samp, int need_depth, int need_distortion,
                                 int need_normal, int track_max_w, int64_t P, int64_t num_rendered,
                                 const int64_t* octree_paths, int levels, const float* vox_centers,
                                 const float* vox_lengths, const float* geos, const float* rgbs, void* geom_buffer,
                                 void* binning_buffer, size_t binning_bytes, void* image_buffer, size_t image_bytes,
                                 float* out_color, float* out_depth, float* out_normal, float* out_T, float* max_w,
                                 int debug, void* stream) {
  int st = svr_rasterize_binning_levels(cam, P, num_rendered, octree_paths, levels, geom_buffer, binning_buffer,
                                        binning_bytes, image_buffer, image_bytes, debug, stream);
  if (st != SVR_OK) return st;
  return svr_rasterize_render(cam, n_samp, need_depth, need_distortion, need_normal, track_max_w, P, num_rendered,
                              vox_centers, vox_lengths, geos, rgbs, geom_buffer, binning_buffer, binning_bytes,
                              image_buffer, image_bytes, out_color, out_depth, out_normal, out_T, max_w, debug,
                              stream);
}

int svr_rasterize_forward(const svr_camera* cam, int n_samp, int need_depth, int need_distortion, int need_normal,
                          int track_max_w, int64_t P, int64_t num_rendered, const int64_t* octree_paths,
                          const float* vox_centers, const float* vox_lengths, const float* geos, const float* rgbs,
                          void* geom_buffer, void* binning_buffer, size_t binning_bytes, void* image_buffer,
                          size_t image_bytes, float* out_color, float* out_depth, float* out_normal, float* out_T,
                          float* max_w, int debug, void* stream) {
  int st = svr_rasterize_binning(cam, P, num_rendered, octree_paths, geom_buffer, binning_buffer, binning_bytes,
                                 image_buffer, image_bytes, debug, stream);
  if (st != SVR_OK) return st;
  return svr_rasterize_render(cam, n_samp, need_depth, need_distortion, need_normal, track_max_w, P, num_rendered,
                              vox_centers, vox_lengths, geos, rgbs, geom_buffer, binning_buffer, binning_bytes,
                              image_buffer, image_bytes, out_color, out_depth, out_normal, out_T, max_w, debug,
                              stream);
}

int svr_rasterize_backward(const svr_camera* cam, int n_samp, int64_t P, int64_t num_rendered,
                           const float* vox_centers, const float* vox_lengths, const float* geos, const float* rgbs,
                           const void* geom_buffer, const void* binning_buffer, const void* image_buffer,
                           const float* out_T, const float* dL_dcolor, const float* dL_ddepth,
                           const float* dL_dnormal, const float* dL_dT, float lambda_R_concen, const float* gt_color,
                           float lambda_ascending, float lambda_dist, int need_depth, int need_normal,
                           const float* out_depth, const float* out_normal, float* dL_dgeos, float* dL_drgbs,
                           float* subdiv_p_bw, int debug, void* stream_) {
  (void)out_normal;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  if (!valid_camera(cam) || n_samp < 1 || n_samp > kMaxSamples || P < 0 || num_rendered < 0) return SVR_ERR_SHAPE;
  if (P == 0) return SVR_OK;
  const bool need_dist = lambda_dist > 0;
  if (!out_T || !dL_dcolor || !dL_dT || !dL_dgeos || !dL_drgbs || !subdiv_p_bw || (need_depth && !dL_ddepth) ||
      (need_normal && !dL_dnormal) || (need_dist && !out_depth) || (lambda_R_concen > 0 && !gt_color))
    return SVR_ERR_SHAPE;
  if (!aligned16(geos)) return SVR_ERR_ALIGN;
  const int W = cam->width, H = cam->height;
  GeomLayout g = geom_layout(const_cast<void*>(geom_buffer), P);
  ImageLayout im = image_layout(const_cast<void*>(image_buffer), W, H);
  BinningLayout bl = binning_layout(const_cast<void*>(binning_buffer), (size_t)num_rendered, 0);
  const ViewParams vp = make_view(*cam);
  VoxelArrays va{g.bbox, vox_centers, vox_lengths, geos, nullptr, rgbs};
  BwdTileIn in{out_T, im.n_contrib, dL_dcolor, need_depth ? dL_ddepth : nullptr,
               need_normal ? dL_dnormal : nullptr, dL_dT, lambda_R_concen > 0 ? gt_color : nullptr,
               need_dist ? out_depth : nullptr, lambda_R_concen, lambda_ascending, lambda_dist, 1};
  BwdTileOut out{dL_dgeos, dL_drgbs, subdiv_p_bw, g.header + 1, aligned16(dL_dgeos) ? 1 : 0};
  // the forward's tile order (read only: the image buffer is the forward's saved state)
  launch_render_bwd(vp, im.ranges, im.tile_last, num_rendered > 0 ? bl.vals_b : nullptr, va, in, out, n_samp,
                    need_depth != 0, need_dist, need_normal != 0, im.order, stream);
  return check_launch(debug, stream);
}

int svr_unpack_image_state(int width, int height, const void* image_buffer, int32_t* ranges, int32_t* tile_last,
                           int32_t* n_contrib, void* stream_) {
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  if (width <= 0 || height <= 0 || !image_buffer) return SVR_ERR_SHAPE;
  ImageLayout im = image_layout(const_cast<void*>(image_buffer), width, height);
  const size_t T = (size_t)tiles_x(width) * tiles_y(height);
  if (ranges) cudaMemcpyAsync(ranges, im.ranges, T * sizeof(uint2), cudaMemcpyDeviceToDevice, stream);
  if (tile_last) cudaMemcpyAsync(tile_last, im.tile_last, T * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream);
  if (n_contrib)
    cudaMemcpyAsync(n_contrib, im.n_contrib, (size_t)width * height * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                    stream);
  return check_launch(0, stream);
}

int svr_binning_sorted_wide(const void* binning_buffer, int64_t num_rendered, int width, int height,
                            const uint64_t** keys_lo, const uint64_t** keys_hi, const uint32_t** vals) {
  if (!binning_buffer || num_rendered < 0 || width <= 0 || height <= 0) return SVR_ERR_SHAPE;
  DeepBinning d = deep_layout(const_cast<void*>(binning_buffer), (size_t)num_rendered,
                              tiles_x(width) * tiles_y(height), nullptr);
  if (keys_lo) *keys_lo = d.keys_lo;
  if (keys_hi) *keys_hi = d.keys_hi;
  if (vals) *vals = d.vals_out;
  return SVR_OK;
}

int svr_binning_sorted(const void* binning_buffer, int64_t num_rendered, int width, int height,
                       const uint64_t** keys, const uint32_t** vals) {
  (void)width;
  (void)height;
  if (!binning_buffer || num_rendered < 0) return SVR_ERR_SHAPE;
  BinningLayout bl = binning_layout(const_cast<void*>(binning_buffer), (size_t)num_rendered, 0);
  if (keys) *keys = bl.keys_b;
  if (vals) *vals = bl.vals_b;
  return SVR_OK;
}

int svr_geom_arrays(const void* geom_buffer, int64_t P, const uint32_t** n_dup, const uint32_t** scan,
                    const uint64_t** bboxes, const uint32_t** quads) {
  if (!geom_buffer || P < 0) return SVR_ERR_SHAPE;
  GeomLayout g = geom_layout(const_cast<void*>(geom_buffer), P);
  if (n_dup) *n_dup = g.ndup;
  if (scan) *scan = g.scan;
  if (bboxes) *bboxes = reinterpret_cast<const uint64_t*>(g.bbox);
  if (quads) *quads = g.quad;
  return SVR_OK;
}

int svr_sh_compute(int degree, int64_t n_idx, const int64_t* idx, int64_t P, int M, const float* vox_centers,
                   const float* cam_pos, const void* sh0, const void* shs, int sh_bf16, float* rgbs, void* stream_) {
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  if (degree < 0 || degree > 3 || P < 0 || n_idx < 0 || M < 1 || (M - 1) < (degree + 1) * (degree + 1) - 1 ||
      (n_idx > 0 && !idx) || P >= (1ll << 31))
    return SVR_ERR_SHAPE;
  if (P == 0) return SVR_OK;
  launch_sh_eval(degree, (int)n_idx, (int)P, M, idx, vox_centers, cam_pos, sh0, shs, sh_bf16 != 0, rgbs, stream);
  return check_launch(0, stream);
}

int svr_sh_compute_bw(int degree, int M, int64_t n_idx, const int64_t* idx, int64_t P, const float* vox_centers,
                      const float* cam_pos, const float* dL_drgbs, float* dL_dsh0, float* dL_dshs, void* stream_) {
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  if (degree < 0 || degree > 3 || P < 0 || n_idx < 0 || M < 1 || (M - 1) < (degree + 1) * (degree + 1) - 1 ||
      (n_idx > 0 && !idx) || P >= (1ll << 31))
    return SVR_ERR_SHAPE;
  if (P == 0) return SVR_OK;
  launch_sh_eval_bw(degree, (int)n_idx, (int)P, M, idx, vox_centers, cam_pos, dL_drgbs, dL_dsh0, dL_dshs, stream);
  return check_launch(0, stream);
}

int svr_unbiased_adam_step(int sparse, int64_t numel, float* param, const float* grad, float* exp_avg,
                           float* exp_avg_sq, double step, double lr, double beta1, double beta2, float eps,
                           void* stream_) {
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  if (numel < 0) return SVR_ERR_SHAPE;
  if (numel == 0) return SVR_OK;
  // Bias corrections in double on the host (adam_step.cu:117-122).
  const double bc1 = 1.0 - pow(beta1, step);
  const double bc2 = 1.0 - pow(beta2, step);
  const double step_size = lr / bc1;
  const double rsqrt_bc2 = 1.0 / sqrt(bc2);
  launch_adam(false, sparse != 0, numel, param, grad, exp_avg, exp_avg_sq, (float)step_size, (float)beta1,
              (float)beta2, (float)rsqrt_bc2, eps, stream);
  return check_launch(0, stream);
}

int svr_biased_adam_step(int sparse, int64_t numel, float* param, const float* grad, float* exp_avg,
                         float* exp_avg_sq, float lr, float beta1, float beta2, float eps, void* stream_) {
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  if (numel < 0) return SVR_ERR_SHAPE;
  if (numel == 0) return SVR_OK;
  launch_adam(true, sparse != 0, numel, param, grad, exp_avg, exp_avg_sq, lr, beta1, beta2, 0.f, eps, stream);
  return check_launch(0, stream);
}

int svr_fused_adam_step(int n_groups, int sparse, void* const* params, const int* param_bf16,
                        const float* const* grads, float* const* exp_avgs, float* const* exp_avg_sqs,
                        const int64_t* numels, const double* steps, const double* lrs, double beta1, double beta2,
                        float eps, void* stream_) {
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  if (n_groups < 0 || n_groups > kMaxAdamGroups) return SVR_ERR_SHAPE;
  AdamGroupTable t;
  memset(&t, 0, sizeof(t));
  t.n = n_groups;
  t.sparse = sparse != 0;
  for (int i = 0; i < n_groups; ++i) {
    if (numels[i] < 0) return SVR_ERR_SHAPE;
    if (!aligned16(grads[i]) || !aligned16(exp_avgs[i]) || !aligned16(exp_avg_sqs[i]) ||
        (reinterpret_cast<uintptr_t>(params[i]) & (param_bf16[i] ? 7u : 15u)))
      return SVR_ERR_ALIGN;
    const double bc1 = 1.0 - pow(beta1, steps[i]);
    const double bc2 = 1.0 - pow(beta2, steps[i]);
    AdamGroup& G = t.g[i];
    G.param = params[i];
    G.param_bf16 = param_bf16[i];
    G.grad = grads[i];
    G.exp_avg = exp_avgs[i];
    G.exp_avg_sq = exp_avg_sqs[i];
    G.numel = numels[i];
    G.step_size = (float)(lrs[i] / bc1);
    G.beta1 = (float)beta1;
    G.beta2 = (float)beta2;
    G.rsqrt_bc2 = (float)(1.0 / sqrt(bc2));
    G.eps = eps;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  launch_adam_fused(t, sms, stream);
  return check_launch(0, stream);
}

int svr_fused_adam_step_device(int n_groups, int sparse, void* const* params, const int* param_bf16,
                               const float* const* grads, float* const* exp_avgs, float* const* exp_avg_sqs,
                               const int64_t* numels, const double* lrs, double beta1, double beta2, float eps,
                               int* d_step, void* stream_) {
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  if (n_groups < 0 || n_groups > kMaxAdamGroups || !d_step) return SVR_ERR_SHAPE;
  AdamGroupTable t;
  memset(&t, 0, sizeof(t));
  t.n = n_groups;
  t.sparse = sparse != 0;
  t.d_step = d_step;
  t.beta1d = beta1;
  t.beta2d = beta2;
  for (int i = 0; i < n_groups; ++i) {
    if (numels[i] < 0) return SVR_ERR_SHAPE;
    if (!aligned16(grads[i]) || !aligned16(exp_avgs[i]) || !aligned16(exp_avg_sqs[i]) ||
        (reinterpret_cast<uintptr_t>(params[i]) & (param_bf16[i] ? 7u : 15u)))
      return SVR_ERR_ALIGN;
    AdamGroup& G = t.g[i];
    G.param = params[i];
    G.param_bf16 = param_bf16[i];
    G.grad = grads[i];
    G.exp_avg = exp_avgs[i];
    G.exp_avg_sq = exp_avg_sqs[i];
    G.numel = numels[i];
    G.lr = lrs[i];
    G.beta1 = (float)beta1;
    G.beta2 = (float)beta2;
    G.eps = eps;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  launch_step_increment(d_step, stream);
  launch_adam_fused(t, sms, stream);
  return check_launch(0, stream);
}

int svr_gather_grid_params(int dim, int64_t n_care, const int64_t* vox_key, const int64_t* care_idx,
                           const float* grid_pts, float* out, void* stream_) {
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  if ((dim != 1 && dim != 3) || n_care < 0 || n_care >= (1ll << 31)) return SVR_ERR_SHAPE;
  launch_gather(dim, (int)n_care, vox_key, care_idx, grid_pts, out, stream);
  return check_launch(0, stream);
}

int svr_gather_grid_params_bw(int dim, int64_t n_care, const int64_t* vox_key, const int64_t* care_idx,
                              const float* dL_dvox, float* dL_dgrid, void* stream_) {
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  if ((dim != 1 && dim != 3) || n_care < 0 || n_care >= (1ll << 31)) return SVR_ERR_SHAPE;
  launch_gather_bw(dim, (int)n_care, vox_key, care_idx, dL_dvox, dL_dgrid, stream);
  return check_launch(0, stream);
}

int svr_gather_grid_geo_all(int64_t P, const int64_t* vox_key, const void* grid_pts, int grid_bf16, void* geos_out,
                            int out_bf16, void* stream_) {
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  if (P < 0 || (P > 0 && (!vox_key || !grid_pts || !geos_out))) return SVR_ERR_SHAPE;
  launch_gather_all_geo(P, vox_key, grid_pts, grid_bf16 != 0, geos_out, out_bf16 != 0, stream);
  return check_launch(0, stream);
}

int svr_scatter_grid_geo_all(int64_t P, const int64_t* vox_key, const float* dL_dgeos, float* dL_dgrid,
                             void* stream_) {
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  if (P < 0 || (P > 0 && (!vox_key || !dL_dgeos || !dL_dgrid))) return SVR_ERR_SHAPE;
  launch_scatter_all_geo(P, vox_key, dL_dgeos, dL_dgrid, stream);
  return check_launch(0, stream);
}

int svr_total_variation_bw(const float* grid_pts, const int64_t* vox_key, float weight, const float* vox_size_inv,
                           int no_tv_s, int tv_sparse, int64_t N, int C, uint8_t* sparse_scratch,
                           float* grid_pts_grad, void* stream_) {
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  if (N < 0 || C < 1 || (N > 0 && (!grid_pts || !vox_key || !grid_pts_grad || (!no_tv_s && !vox_size_inv))) ||
      (tv_sparse && N > 0 && !sparse_scratch))
    return SVR_ERR_SHAPE;
  launch_total_variation_bw(grid_pts, vox_key, weight, vox_size_inv, no_tv_s != 0, tv_sparse ? sparse_scratch : nullptr,
                            N, C, grid_pts_grad, stream);
  return check_launch(0, stream);
}

int svr_read_error(uint32_t* device_word, uint32_t* host_value, void* stream_) {
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  uint32_t v = 0;
  if (cudaMemcpyAsync(&v, device_word, sizeof(v), cudaMemcpyDeviceToHost, stream) != cudaSuccess) return SVR_ERR_CUDA;
  if (cudaStreamSynchronize(stream) != cudaSuccess) return SVR_ERR_CUDA;
  cudaMemsetAsync(device_word, 0, sizeof(uint32_t), stream);
  if (host_value) *host_value = v;
  return v ? SVR_ERR_DEVICE : SVR_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Scratch-free variant of svr_rasterize_preprocess.
//
// For callers that cannot allocate device memory at all (a renderer embedded
// in a host application whose allocator owns every device buffer, code running
// inside a CUDA-graph capture, or a real-time loop that forbids cudaMalloc).
// The only scratch of the projection + scan sequence -- the per-CTA partial
// sums of the scan -- lives in the file-scope device array below instead of
// in the caller's geom buffer.  It bounds P to kNoAllocMaxVoxels.
//
// The array is a host-side stand-in in host code, not a device address: its
// device address is taken with cudaGetSymbolAddress once per device, by the
// first call made with that device current (so that first call should come
// before any stream capture; a lookup that fails is retried by the next
// call).  Every call shares the array: calls that overlap on the GPU (two
// streams, or two threads) race on it.  Nothing in it needs clearing between
// calls: each call writes every partial sum it later reads.
// ---------------------------------------------------------------------------
namespace {

// One 64-bit partial sum per scan CTA of kScanTile voxels (svr_kernels.h),
// plus the alignment slack scan_temp_bytes() reserves.
constexpr int64_t kNoAllocMaxBlocks = 16384;
constexpr int64_t kNoAllocMaxVoxels = (int64_t)kScanTile * kNoAllocMaxBlocks;  // 67,108,864
constexpr int64_t kNoAllocWords = kNoAllocMaxBlocks + 1 + 256 / sizeof(unsigned long long);

__device__ __align__(256) unsigned long long g_noalloc_scan_partials[kNoAllocWords];

constexpr int kNoAllocMaxDevices = 64;
// Device address of the array per device, set once a lookup succeeds; a
// failed lookup (made during a stream capture, say) leaves it null, and the
// next call on that device tries again.
std::atomic<void*> g_noalloc_ptr[kNoAllocMaxDevices];

// Device address of the partial-sum array on the current device.
void* noalloc_scratch(int& status) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) {
    status = SVR_ERR_CUDA;
    return nullptr;
  }
  void* ptr = g_noalloc_ptr[dev].load(std::memory_order_acquire);
  if (!ptr) {
    if (cudaGetSymbolAddress(&ptr, g_noalloc_scan_partials) != cudaSuccess || !ptr) {
      cudaGetLastError();  // clear it, so that a later launch check does not report it again
      status = SVR_ERR_CUDA;
      return nullptr;
    }
    g_noalloc_ptr[dev].store(ptr, std::memory_order_release);
  }
  status = SVR_OK;
  return ptr;
}

}  // namespace

extern "C" int svr_rasterize_preprocess_noalloc(const svr_camera* cam, int64_t P, const int64_t* octree_paths,
                                                const float* vox_centers, const float* vox_lengths,
                                                int32_t* out_n_duplicates, void* geom_buffer, size_t geom_bytes,
                                                int debug, void* stream_) {
  (void)octree_paths;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  if (P < 0 || P >= (1ll << kVoxIdBits) || !valid_camera(cam)) return SVR_ERR_SHAPE;
  if (P > kNoAllocMaxVoxels || scan_temp_bytes((size_t)P) > sizeof(g_noalloc_scan_partials)) return SVR_ERR_CAPACITY;
  if (P == 0) return SVR_OK;
  GeomLayout g = geom_layout(geom_buffer, P);
  if (!geom_buffer || geom_bytes < g.bytes || !vox_centers || !vox_lengths || !out_n_duplicates) return SVR_ERR_SHAPE;
  int st = SVR_OK;
  void* partials = noalloc_scratch(st);
  if (st != SVR_OK) return st;
  ViewTable vt;
  vt.n = 1;
  vt.v[0] = make_view(*cam);
  cudaMemsetAsync(g.header, 0, 16 * sizeof(uint32_t), stream);
  launch_preprocess(vt, (int)P, vox_centers, vox_lengths, out_n_duplicates, g.ndup, g.bbox, g.quad, stream);
  launch_scan_inclusive(g.ndup, g.scan, (size_t)P, partials, g.header, 0xffffffffull, g.header + 1, stream);
  return check_launch(debug, stream);
}

extern "C" int64_t svr_noalloc_max_voxels(void) { return kNoAllocMaxVoxels; }
