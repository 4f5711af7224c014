/*
 * svr_b200.h -- C ABI of the sm_100a sparse-voxel rasterizer (libsvr_b200.so).
 *
 * Drop-in replacement, at the native boundary, for the pybind11 module `_C`
 * of the SVRaster CUDA backend (panicPaul/sv_raster, backends/cuda/binding.cpp:24-55).
 * Each entry point below names the reference function it replaces.  The
 * differences of convention are:
 *   - the caller owns all memory: outputs and opaque state buffers are
 *     allocated by the caller (sizes from the *_bytes queries) and passed as
 *     raw device pointers; every output a reference op returns zero-filled
 *     must be zero-filled by the caller (the Python layer does this);
 *   - every call takes a cudaStream_t (as void*) and enqueues on it; no call
 *     synchronises the device unless `debug` is set;
 *   - every call returns an int status (SVR_OK ...); device-side consistency
 *     failures (the reference __trap()s) set bits of a device error word that
 *     svr_read_error reads.
 * No torch types appear in any signature.
 */
#ifndef SVR_B200_H_
#define SVR_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SVR_OK 0
#define SVR_ERR_SHAPE 1
#define SVR_ERR_CAPACITY 2
#define SVR_ERR_KEYBITS 3
#define SVR_ERR_CUDA 4
#define SVR_ERR_DEVICE 5
#define SVR_ERR_ALIGN 6

/* Compile-time constants (config.h:16,21,23; exported at binding.cpp:51-53). */
int svr_max_num_levels(void);     /* 16 */
float svr_step_sz_scale(void);    /* 100 */
int svr_max_n_samp(void);         /* 3 */
const char* svr_status_string(int status);
int svr_version(void);

/* One pinhole camera.  w2c / c2w are DEVICE pointers to row-major 4x4 float
 * matrices (the reference reads the first 12 entries in-kernel too:
 * preprocess.cu:57-60, forward.cu:103-109). */
typedef struct svr_camera {
  int width, height;
  float tanfovx, tanfovy;
  float cx, cy;
  const float* w2c;
  const float* c2w;
  float near_plane;
  float bg_color;
} svr_camera;

/* ---- opaque state buffer sizes (raster_state.cu:54-117) ---------------- */
size_t svr_geom_buffer_bytes(int64_t P);
size_t svr_image_buffer_bytes(int width, int height);
size_t svr_binning_buffer_bytes(int64_t num_rendered, int width, int height);

/* Replaces PREPROCESS::rasterize_preprocess (preprocess.cu:136-199, binding
 * "rasterize_preprocess").  Writes out_n_duplicates[P] (int32) and fills the
 * caller's geom buffer.  It also scans the duplicate counts on the device and
 * stores the instance count (uint32) at svr_geom_count_ptr(geom). */
int svr_rasterize_preprocess(const svr_camera* cam, int64_t P, const int64_t* octree_paths,
                             const float* vox_centers, const float* vox_lengths, int32_t* out_n_duplicates,
                             void* geom_buffer, size_t geom_bytes, int debug, void* stream);

/* svr_rasterize_preprocess whose scan scratch lives inside the library.  No
 * counterpart in the reference.  For callers that cannot allocate device
 * memory (an embedding host that owns every device buffer, code inside CUDA
 * graph capture, real-time loops): the scan's partial sums live in a static
 * device array of the library, so P is limited to svr_noalloc_max_voxels()
 * (67,108,864); larger P returns SVR_ERR_CAPACITY.  Same arguments and
 * outputs as svr_rasterize_preprocess, and the geom buffer is sized the same
 * way (svr_geom_buffer_bytes): its layout is shared with the other calls, so
 * the scratch region it reserves stays unused here.  The first call on a
 * device looks up the array's device address (make it before any stream
 * capture; a failed lookup is retried by the next call).  All calls share
 * the array: calls that overlap on the GPU race.  The function allocates
 * nothing. */
int svr_rasterize_preprocess_noalloc(const svr_camera* cam, int64_t P, const int64_t* octree_paths,
                                     const float* vox_centers, const float* vox_lengths, int32_t* out_n_duplicates,
                                     void* geom_buffer, size_t geom_bytes, int debug, void* stream);
int64_t svr_noalloc_max_voxels(void);

/* Device address of the uint32 instance count ("num_rendered", read back by
 * the reference at forward.cu:652-658) inside a geom buffer. */
const uint32_t* svr_geom_count_ptr(const void* geom_buffer);
/* Device address of the uint32 device error word inside a geom buffer. */
uint32_t* svr_geom_error_ptr(void* geom_buffer);

/* Replaces FORWARD::rasterize_voxels (forward.cu:739-825, binding
 * "rasterize_voxels") after its count read-back: duplication, sort, tile
 * ranges and compositing.  `num_rendered` is the value at
 * svr_geom_count_ptr(geom).  Outputs (caller-zeroed): out_color [3,H,W],
 * out_depth [3,H,W] (if need_depth || need_distortion, else NULL),
 * out_normal [3,H,W] (if need_normal), out_T [1,H,W], max_w [P] (if
 * track_max_w).  geos and rgbs are fp32 [P,8] and [P,3]. */
int svr_rasterize_forward(const svr_camera* cam, int n_samp_per_vox, int need_depth, int need_distortion,
                          int need_normal, int track_max_w, int64_t P, int64_t num_rendered,
                          const int64_t* octree_paths, const float* vox_centers, const float* vox_lengths,
                          const float* geos, const float* rgbs, void* geom_buffer, void* binning_buffer,
                          size_t binning_bytes, void* image_buffer, size_t image_bytes, float* out_color,
                          float* out_depth, float* out_normal, float* out_T, float* max_w, int debug, void* stream);

/* Octrees 21 levels deep: the forward of the reference's new_cuda backend
 * (backends/new_cuda/src/forward.cu:660-752, config.h:16,24-34), whose
 * 63-bit Morton ranks make the (tile, rank) sort key 128 bits wide
 * (auxiliary.h:17-25,66-87).  levels = 16 is svr_rasterize_forward; levels =
 * 21 sorts by (tile, 63-bit rank) -- the same order as the reference's stable
 * wide-key sort -- and leaves the sorted values and tile ranges where
 * svr_rasterize_backward reads them.  The binning buffer is sized by
 * svr_binning_buffer_bytes_levels. */
size_t svr_binning_buffer_bytes_levels(int64_t num_rendered, int width, int height, int levels);
int svr_rasterize_binning_levels(const svr_camera* cam, int64_t P, int64_t num_rendered, const int64_t* octree_paths,
                                 int levels, void* geom_buffer, void* binning_buffer, size_t binning_bytes,
                                 void* image_buffer, size_t image_bytes, int debug, void* stream);
int svr_rasterize_forward_levels(const svr_camera* cam, int n_samp_per_vox, int need_depth, int need_distortion,
                                 int need_normal, int track_max_w, int64_t P, int64_t num_rendered,
                                 const int64_t* octree_paths, int levels, const float* vox_centers,
                                 const float* vox_lengths, const float* geos, const float* rgbs, void* geom_buffer,
                                 void* binning_buffer, size_t binning_bytes, void* image_buffer, size_t image_bytes,
                                 float* out_color, float* out_depth, float* out_normal, float* out_T, float* max_w,
                                 int debug, void* stream);

/* The two stages of svr_rasterize_forward, callable separately (same
 * arguments): duplication + sort + tile ranges (forward.cu:660-700), then the
 * compositing kernel alone (forward.cu:702-731).  The render stage also ranks
 * the tiles by list length and stores that work order in the image buffer;
 * its compositing launch and the backward's run the largest tiles first
 * (results do not depend on the order). */
int svr_rasterize_binning(const svr_camera* cam, int64_t P, int64_t num_rendered, const int64_t* octree_paths,
                          void* geom_buffer, void* binning_buffer, size_t binning_bytes, void* image_buffer,
                          size_t image_bytes, int debug, void* stream);
int svr_rasterize_render(const svr_camera* cam, int n_samp_per_vox, int need_depth, int need_distortion,
                         int need_normal, int track_max_w, int64_t P, int64_t num_rendered, const float* vox_centers,
                         const float* vox_lengths, const float* geos, const float* rgbs, void* geom_buffer,
                         void* binning_buffer, size_t binning_bytes, void* image_buffer, size_t image_bytes,
                         float* out_color, float* out_depth, float* out_normal, float* out_T, float* max_w, int debug,
                         void* stream);

/* Replaces BACKWARD::rasterize_voxels_backward (backward.cu:655-769, binding
 * "rasterize_voxels_backward").  Outputs (caller-zeroed): dL_dgeos [P,8],
 * dL_drgbs [P,3], subdiv_p_bw [P,1].  dL_ddepth / dL_dnormal / gt_color /
 * out_depth / out_normal may be NULL when the matching feature is off. */
int svr_rasterize_backward(const svr_camera* cam, int n_samp_per_vox, int64_t P, int64_t num_rendered,
                           const float* vox_centers, const float* vox_lengths, const float* geos, const float* rgbs,
                           const void* geom_buffer, const void* binning_buffer, const void* image_buffer,
                           const float* out_T, const float* dL_dcolor, const float* dL_ddepth,
                           const float* dL_dnormal, const float* dL_dT, float lambda_R_concen, const float* gt_color,
                           float lambda_ascending, float lambda_dist, int need_depth, int need_normal,
                           const float* out_depth, const float* out_normal, float* dL_dgeos, float* dL_drgbs,
                           float* subdiv_p_bw, int debug, void* stream);

/* Replaces RASTER_STATE::unpack_ImageState (raster_state.cu:155-175):
 * copies ranges [T,2], tile_last [T], n_contrib [H*W] (int32, device) out of
 * an image buffer. */
int svr_unpack_image_state(int width, int height, const void* image_buffer, int32_t* ranges, int32_t* tile_last,
                           int32_t* n_contrib, void* stream);
/* Sorted instance keys/values of a binning buffer (device pointers), for
 * parity checks of the sort (forward.cu:681-686 results). */
int svr_binning_sorted(const void* binning_buffer, int64_t num_rendered, int width, int height,
                       const uint64_t** keys, const uint32_t** vals);
/* The same for a 21-level binning buffer: the sorted 128-bit keys as their
 * low and high words (the reference's SortKey128 {hi, lo}: lo = tile << 63 |
 * rank, hi = tile >> 1) and the sorted values. */
int svr_binning_sorted_wide(const void* binning_buffer, int64_t num_rendered, int width, int height,
                            const uint64_t** keys_lo, const uint64_t** keys_hi, const uint32_t** vals);
/* Per-voxel preprocess state of a geom buffer (device pointers). */
int svr_geom_arrays(const void* geom_buffer, int64_t P, const uint32_t** n_dup, const uint32_t** scan,
                    const uint64_t** bboxes, const uint32_t** quads);

/* Replaces SH_COMPUTE::sh_compute (sh_compute.cu:244-270).  rgbs [P,3]
 * caller-zeroed; idx may be NULL with n_idx = 0 (all voxels).  sh0 [P,3],
 * shs [P,M-1,3]; coefficient storage fp32 or bf16 (sh_bf16 = 1). */
int svr_sh_compute(int degree, int64_t n_idx, const int64_t* idx, int64_t P, int M, const float* vox_centers,
                   const float* cam_pos, const void* sh0, const void* shs, int sh_bf16, float* rgbs, void* stream);
/* Replaces SH_COMPUTE::sh_compute_bw (sh_compute.cu:272-299).  dL_dsh0 [P,3],
 * dL_dshs [P,M-1,3] caller-zeroed. */
int svr_sh_compute_bw(int degree, int M, int64_t n_idx, const int64_t* idx, int64_t P, const float* vox_centers,
                      const float* cam_pos, const float* dL_drgbs, float* dL_dsh0, float* dL_dshs, void* stream);

/* Replace ADAM_STEP::unbiased_adam_step / biased_adam_step
 * (adam_step.cu:106-158); `step` is the 1-based step count. */
int svr_unbiased_adam_step(int sparse, int64_t numel, float* param, const float* grad, float* exp_avg,
                           float* exp_avg_sq, double step, double lr, double beta1, double beta2, float eps,
                           void* stream);
int svr_biased_adam_step(int sparse, int64_t numel, float* param, const float* grad, float* exp_avg,
                         float* exp_avg_sq, float lr, float beta1, float beta2, float eps, void* stream);

/* Fused multi-group unbiased Adam: one launch for up to 8 groups (no
 * reference counterpart; same per-element arithmetic as
 * unbiased_adam_step_cuda_kernel, adam_step.cu:28-64).  Arrays must be
 * 16-byte aligned; params may be fp32 or bf16 (param_bf16[i] = 1). */
int svr_fused_adam_step(int n_groups, int sparse, void* const* params, const int* param_bf16,
                        const float* const* grads, float* const* exp_avgs, float* const* exp_avg_sqs,
                        const int64_t* numels, const double* steps, const double* lrs, double beta1, double beta2,
                        float eps, void* stream);

/* The same with the step count kept on the device: *d_step is incremented
 * on the stream and the bias correction computed from it on the device, so a
 * captured training step replays with an advancing step (no reference
 * counterpart). */
int svr_fused_adam_step_device(int n_groups, int sparse, void* const* params, const int* param_bf16,
                               const float* const* grads, float* const* exp_avgs, float* const* exp_avg_sqs,
                               const int64_t* numels, const double* lrs, double beta1, double beta2, float eps,
                               int* d_step, void* stream);

/* Replace GEO_PARAMS_GATHER::gather_triinterp_geo_params(_bw) and the feat
 * variants (geo_params_gather.cu:134-222).  dim = 1 (geo) or 3 (feat). */
int svr_gather_grid_params(int dim, int64_t n_care, const int64_t* vox_key, const int64_t* care_idx,
                           const float* grid_pts, float* out, void* stream);
int svr_gather_grid_params_bw(int dim, int64_t n_care, const int64_t* vox_key, const int64_t* care_idx,
                              const float* dL_dvox, float* dL_dgrid, void* stream);
/* The grid-point gather of every voxel (GatherGeoParams with all voxels
 * cared for, renderer.py:319-345, geo_params_gather.cu:22-46): geos_out[p,c] =
 * grid_pts[vox_key[p,c]], grid and output each fp32 or bf16 -- the density
 * input of the batched step when training grid points.  vox_key int64 [P,8]. */
int svr_gather_grid_geo_all(int64_t P, const int64_t* vox_key, const void* grid_pts, int grid_bf16, void* geos_out,
                            int out_bf16, void* stream);
/* Its backward (geo_params_gather.cu:48-72 for all voxels): adds dL_dgeos
 * [P,8] fp32 into dL_dgrid [M] fp32 at vox_key. */
int svr_scatter_grid_geo_all(int64_t P, const int64_t* vox_key, const float* dL_dgeos, float* dL_dgrid,
                             void* stream);

/* Replaces TV_COMPUTE::total_variation_bw (tv_compute.cu:84-110): adds the
 * total-variation gradient of grid_pts [M,C] over the N voxels' 8 corners
 * (vox_key [N,8]) into grid_pts_grad in place.  tv_sparse needs a caller
 * scratch of N*C bytes; the sparse test uses the gradient as it was before
 * the call (the reference's reads race with its own updates). */
int svr_total_variation_bw(const float* grid_pts, const int64_t* vox_key, float weight, const float* vox_size_inv,
                           int no_tv_s, int tv_sparse, int64_t N, int C, uint8_t* sparse_scratch,
                           float* grid_pts_grad, void* stream);

/* Read and clear a device error word (synchronises `stream`). */
int svr_read_error(uint32_t* device_word, uint32_t* host_value, void* stream);

/* ---- multi-view batched path ------------------------------------------
 * No reference counterpart: the reference renders one view per call and
 * reads the instance count back to the host (forward.cu:601-734).
 * N <= 64 views share one voxel set.  Per-view image arrays are laid out view
 * after view: colour [sum_v 3*H_v*W_v] (each view planar [3,H,W]), T and
 * dL_dT [sum_v H_v*W_v].  The plan fixes camera sizes and the DEVICE
 * addresses of every view's w2c/c2w (their contents may change between
 * calls); the workspace is caller-allocated (svr_batch_plan_create reports its
 * size).  Nothing synchronises: an instance count above `capacity` sets
 * SVR_DEVERR_CAPACITY (0x4) in the error word and leaves outputs invalid; the
 * total instance count is at svr_batch_count_ptr.  Every voxel's octree level
 * must be <= max_level (checked on the device: SVR_DEVERR_LEVEL, 0x10). */
typedef struct svr_batch_plan svr_batch_plan;
/* tile_size: compositing tiles of 8x8, 16x16 (the reference's) or 32x32
 * pixels.  Images, T and per-view gradients are the same for every tile size
 * (a pixel sees the same instances in the same order); the instance count,
 * tile lists and contributor indices are those of the chosen tiling. */
int svr_batch_plan_create(int n_views, const svr_camera* cams, int64_t P, int64_t capacity, int n_samp_per_vox,
                          int max_level, int tile_size, svr_batch_plan** plan, size_t* workspace_bytes);
void svr_batch_plan_destroy(svr_batch_plan* plan);
/* The plan ranks every (voxel, quadrant) pair once, on the first
 * svr_batch_prepare, from the octree paths it is given (one radix sort of 8P
 * keys); instances are then keyed by that rank position.  The table is
 * rebuilt when prepare sees a different octree_paths pointer or after this
 * call (for paths changed in place). */
int svr_batch_plan_invalidate_geometry(svr_batch_plan* plan);
/* Compositing schedule of svr_batch_render / svr_batch_backward: both are
 * persistent launches that take (view, tile) items from a device counter.
 * order_flags bit 0 (forward) / bit 1 (backward), both set by default, rank
 * the tiles largest first (by instance count, eighth-octave buckets) before
 * the launch; a clear bit keeps tile order.  The ctas_per_sm caps (0 = as
 * many as fit, the default) bound the resident CTAs per SM.  Results do not
 * depend on the schedule (gradients only up to the order of floating-point
 * additions). */
int svr_batch_plan_set_schedule(svr_batch_plan* plan, int order_flags, int fwd_ctas_per_sm, int bwd_ctas_per_sm);
/* Segment-size buckets of the per-tile segment sort in svr_batch_prepare:
 * tiles of at most small_n (256, 512 or 1024) instances are sorted by one
 * small CTA each, longer ones in runs of `chunk` (2048 or 4096) instances
 * merged afterwards.  Defaults 512 / 4096; the order is the same for all. */
int svr_batch_plan_set_sort_buckets(svr_batch_plan* plan, int small_n, int chunk);
/* How svr_batch_prepare groups the instances by tile before the per-tile
 * segment sort: 1 (default) a counting sort (per-tile counts, their scan,
 * one scatter pass with one atomic per tile per warp), 0 LSD radix passes
 * over the tile bits of the keys.  The sorted lists are the same for both. */
int svr_batch_plan_set_binning(svr_batch_plan* plan, int binning);
/* Records staged into shared memory per round by the compositing kernels:
 * 128, 256 (default) or 512 with 16x16 tiles, 32, 64 (default) or 128 with
 * 8x8, 256 with 32x32. */
int svr_batch_plan_set_staging(svr_batch_plan* plan, int records);
/* The backward's staging depth alone (same values; set_staging sets both):
 * the backward keeps more per-record state in shared memory than the forward,
 * so its best depth can be smaller. */
int svr_batch_plan_set_backward_staging(svr_batch_plan* plan, int records);
int svr_batch_plan_tile_size(const svr_batch_plan* plan);
/* Backward gradient reduction inside a warp: a staged record's 12 gradient
 * values from at most atomic_lanes (1-32, default 1) contributing lanes are
 * added to its shared accumulator with atomics, from up to 8 lanes by a
 * transposition through shared memory, from more lanes through a 13-shuffle
 * reduce-scatter.  Configurations that keep a slot per warp (at most two
 * warps, 32 staged records) store one lane's values directly whatever the
 * setting.  Only the order of additions changes. */
int svr_batch_plan_set_reduction(svr_batch_plan* plan, int atomic_lanes);
/* Arithmetic of the compositing loops of svr_batch_render / svr_batch_backward.
 * exact = 1: the reference's operations (forward.cu:243-253, backward.cu:309-333:
 * libdevice expf, IEEE division); images, T and contributor counts are
 * bit-identical to svr_rasterize_render's.  exact = 0 (default): the hardware
 * exponential and an approximate division (a few ulp each) for the
 * per-(pixel, voxel) exponentials and the transmittance recovery -- fewer
 * instructions in both loops; images and gradients then agree with the exact
 * form to fp32 accumulation error (a pixel may stop one voxel earlier or later
 * where its transmittance lands on the 1e-4 early-stop threshold). */
int svr_batch_plan_set_arithmetic(svr_batch_plan* plan, int exact);
/* Pixel bbox of each (view, voxel) pair written by svr_batch_prepare.
 * culling = 0: the reference's bbox, each side of the projected corners'
 * extent rounded to the nearest pixel (preprocess.cu:98-113); tile lists and
 * contributor counts are the plain path's.  culling = 1: the pixels of that
 * bbox whose centre lies within 0.05 pixel of the unrounded extent, for voxels
 * with all 8 corners in front of the near plane -- every other pixel's ray
 * provably misses the cube, so the lists lose instances that contribute
 * nothing; a voxel left with no pixel centre is culled for that view (n_dup 0).
 * Images, T and gradients are unchanged; contributor counts (list positions)
 * shrink.  culling = -1 (default): 1 with the fast arithmetic, 0 with the
 * exact one. */
int svr_batch_plan_set_culling(svr_batch_plan* plan, int culling);
/* Pixels per thread of the compositing kernels: 1 (default) or 2 (a warp
 * covers an 8x8 block, each lane two pixels four rows apart; a record's
 * shared-memory fields are read once for both and, in the backward, one warp
 * reduction serves both).  Used with 8x8 tiles staging 32 or 64 records and
 * 16x16 tiles staging 128 or 256; other tile configurations run one pixel
 * per thread.  Images, T and contributor counts do not depend on it. */
int svr_batch_plan_set_pixels_per_thread(svr_batch_plan* plan, int pixels);
/* Pixels per thread of svr_batch_backward alone: 1 or 2, or 0 to follow
 * svr_batch_plan_set_pixels_per_thread (default).  The forward walks each
 * pixel's own records with one pixel per thread, while the backward's warp
 * reduction favours two, so the best choices can differ. */
int svr_batch_plan_set_backward_pixels_per_thread(svr_batch_plan* plan, int pixels);
int64_t svr_batch_plan_pixels(const svr_batch_plan* plan);
int64_t svr_batch_plan_tiles(const svr_batch_plan* plan);
int svr_batch_plan_groups(const svr_batch_plan* plan);
const uint32_t* svr_batch_count_ptr(const svr_batch_plan* plan, const void* workspace);
uint32_t* svr_batch_error_ptr(const svr_batch_plan* plan, void* workspace);
/* Packed pixel bbox of every (view, voxel) pair [V,P] (uint2 as uint64:
 * .x = xmin << 16 | ymin, .y = xmax << 16 | ymax), valid after prepare. */
const uint64_t* svr_batch_bbox_ptr(const svr_batch_plan* plan, const void* workspace);
/* Device arrays inside a workspace: rgbs [V,P,3], drgbs [V,P,4] (dL/drgb in
 * xyz, the subdivision priority in w), ranges [T] (uint2 as uint64),
 * tile_last [T], n_contrib [pixels], n_dup [V,P], sorted values. */
int svr_batch_arrays(const svr_batch_plan* plan, const void* workspace, const float** rgbs, const float** drgbs,
                     const uint64_t** ranges, const uint32_t** tile_last, const uint32_t** n_contrib,
                     const uint32_t** n_dup, const uint32_t** sorted_vals);
/* Projection fused with SH colour (fp32 or bf16 coefficients, degree 0-3),
 * scan, duplication, grouped sort and tile ranges of every view. */
int svr_batch_prepare(svr_batch_plan* plan, void* workspace, const int64_t* octree_paths, const float* vox_centers,
                      const float* vox_lengths, const void* sh0, const void* shs, int sh_bf16, int sh_degree, int M,
                      void* stream);
/* Compositing of every (view, tile) in one persistent launch; geos fp32 or bf16 [P,8].
 * Every pixel of out_color / out_T is written.  Reads the tile lists of the
 * last svr_batch_prepare on this workspace (call prepare first). */
int svr_batch_render(svr_batch_plan* plan, void* workspace, const float* vox_centers, const float* vox_lengths,
                     const void* geos, int geos_bf16, float* out_color, float* out_T, void* stream);
/* Recompute-backward of every (view, tile) in one persistent launch:
 * dL_dgeos [P,8] summed over views (caller-zeroed, 16-byte aligned rows: it
 * is accumulated with vector reductions); per-view dL/drgb and subdivision
 * priority kept in the workspace for svr_batch_sh_backward. */
int svr_batch_backward(svr_batch_plan* plan, void* workspace, const float* vox_centers, const float* vox_lengths,
                       const void* geos, int geos_bf16, const float* out_T, const float* dL_dcolor,
                       const float* dL_dT, float* dL_dgeos, void* stream);
/* svr_batch_render / svr_batch_backward with the densities as grid points:
 * corner c of voxel p is grid[vox_key[8 p + c]] (vox_key int64 [P,8], grid
 * fp32 or bf16 [M]), read while each record is staged, and the backward adds
 * every record's corner gradients straight into dL_dgrid (fp32 [M],
 * accumulated: zero it first) -- GatherGeoParams and its backward
 * (renderer.py:319-345, geo_params_gather.cu:22-72) fused into the staging
 * and the flush.  The results equal svr_gather_grid_geo_all + svr_batch_render
 * / svr_batch_backward + svr_scatter_grid_geo_all (images bitwise; gradients
 * to the order of additions).  The grid reads and atomics are per (voxel,
 * tile) instead of per voxel, so the separate gather and scatter cost less
 * (measured 3 % with one view per step, 8 % with eight). */
int svr_batch_render_grid(svr_batch_plan* plan, void* workspace, const float* vox_centers, const float* vox_lengths,
                          const int64_t* vox_key, const void* grid, int grid_bf16, float* out_color, float* out_T,
                          void* stream);
int svr_batch_backward_grid(svr_batch_plan* plan, void* workspace, const float* vox_centers,
                            const float* vox_lengths, const int64_t* vox_key, const void* grid, int grid_bf16,
                            const float* out_T, const float* dL_dcolor, const float* dL_dT, float* dL_dgrid,
                            void* stream);
/* dL/dsh0 [P,3] and dL/dshs [P,M-1,3] summed over views (overwritten), and,
 * when subdiv is not null, the subdivision priority subdiv_p_bw [P] summed
 * over views (overwritten; backward.cu:514 per view). */
int svr_batch_sh_backward(svr_batch_plan* plan, void* workspace, const float* vox_centers, int sh_degree, int M,
                          float* dL_dsh0, float* dL_dshs, float* subdiv, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SVR_B200_H_ */
