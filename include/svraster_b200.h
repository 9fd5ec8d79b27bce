/*
 * svraster_b200 -- C ABI of the B200 (sm_100a) sparse-voxel SDF rasterizer.
 *
 * Plain pointers, sizes and a CUDA stream (passed as void*); no framework types.  Every
 * pointer argument is a DEVICE pointer unless its name ends in _host.  Every entry point
 * returns 0 on success or a negative svr_status_t; svr_last_error() gives a message.
 * Launches are asynchronous on `stream` unless noted.  Entry points that size their work
 * from device data (svr_count_rendered, svr_valid_table_count) synchronise `stream`.
 *
 * The functions replace the native ops of the reference's `svraster_cuda._C` module
 * (cuda/binding.cpp:28-56); each declaration names the reference function it stands for.
 */
#ifndef SVRASTER_B200_H
#define SVRASTER_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define SVR_API __attribute__((visibility("default")))
#else
#define SVR_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    SVR_OK = 0,
    SVR_ERR_ARG = -1,        /* bad argument (size, mode, null pointer)            */
    SVR_ERR_CUDA = -2,       /* a CUDA runtime call failed                          */
    SVR_ERR_CAPACITY = -3,   /* a caller-provided buffer is too small               */
    SVR_ERR_DEVICE = -4,     /* a kernel reported an error through its status word  */
    SVR_ERR_UNSUPPORTED = -5 /* mode not supported by this build                    */
} svr_status_t;

/* One camera.  A batch of views is an array of these; views are rendered into packed
 * outputs where view v owns pixels [pix_offset, pix_offset + W*H) of every plane and
 * tiles [tile_offset, tile_offset + tiles_x*tiles_y) of the tile arrays.
 * Matches RasterSettings (cuda/svraster_cuda/renderer.py:16-41): w2c / c2w are row-major
 * 4x4 float32 device matrices of which the first 3 rows are used; bg is 3 floats. */
typedef struct {
    int32_t width, height;
    int32_t tiles_x, tiles_y;
    int32_t tile_offset;
    int32_t pad0;
    int64_t pix_offset;
    float tanfovx, tanfovy, cx, cy;
    float near_plane;
    float pad1;
    const float* w2c;
    const float* c2w;
    const float* bg;
} svr_view_t;

/* Maximum number of views in one batched launch. */
#define SVR_MAX_VIEWS 128
#define SVR_TILE 16

SVR_API const char* svr_last_error(void);
SVR_API int svr_version(void);
/* Number of this library's own kernels launched by this process so far (no counterpart in
 * the reference; used to report launches inside a timed region). */
SVR_API long long svr_kernel_launches(void);

/* ---------------------------------------------------------------- preprocess
 * Replaces _C.rasterize_preprocess (cuda/src/preprocess.cu:158-228).
 * Per view v and voxel i writes n_dup[v*N + i] (int32) and the view's geometry state into
 * geom_buffer (svr_geom_buffer_bytes(N * n_views) bytes, 256-aligned device memory). */
SVR_API size_t svr_geom_buffer_bytes(int64_t n_items);
SVR_API int svr_preprocess(const svr_view_t* views_host, int n_views, int N,
                   const float* centers, const float* lengths, const uint8_t* is_leaf,
                   const int64_t* octpaths,
                   int32_t* out_n_dup, void* geom_buffer, void* stream);

/* Read the per-voxel geometry fields back out of a geom buffer (for tests and
 * reference-compatible debugging): n_dup u32[M], bboxes u32[M,2], quadrant bits u32[M]. */
SVR_API int svr_unpack_geom(const void* geom_buffer, int64_t n_items, uint32_t* n_dup, uint32_t* bboxes,
                    uint32_t* bits, void* stream);

/* Prefix-sum the duplication counts and return the total number of (tile, voxel, octant)
 * records R and the OR of the octree paths of every rendered voxel (used to trim the
 * sort key).  Synchronises `stream` (the reference does the same, forward.cu:892-896). */
SVR_API int svr_count_rendered(int64_t n_items, void* geom_buffer, int64_t* num_rendered_host,
                       uint64_t* path_or_host, void* stream);

/* The prefix sum of svr_count_rendered without the read-back or the synchronisation (no
 * counterpart in the reference): for a step captured into a CUDA graph, which bins into a
 * buffer of fixed capacity and never learns the record total on the host. */
SVR_API int svr_scan_rendered(int64_t n_items, void* geom_buffer, void* stream);

/* ---------------------------------------------------------------- binning
 * Replaces the duplicate/sort/range part of rasterize_voxels_procedure
 * (cuda/src/forward.cu:749-829, 882-939): emits (tile | order-rank, octant | voxel) pairs,
 * sorts them with a stable radix sort whose key is trimmed to the bits that can differ
 * (order-equivalent to the reference's 64-bit key), and writes per-tile [start, end). */
SVR_API size_t svr_binning_buffer_bytes(int64_t num_rendered, int total_tiles);
SVR_API size_t svr_image_buffer_bytes(int64_t total_pixels, int total_tiles);
SVR_API int svr_bin_and_sort(const svr_view_t* views_host, int n_views, int N, int64_t num_rendered,
                     uint64_t path_or, const int64_t* octpaths, void* geom_buffer,
                     void* binning_buffer, size_t binning_bytes, void* image_buffer, void* stream);
/* num_rendered above (and in the render calls) is the capacity of the binning buffer: the
 * record total from svr_count_rendered, or any bound on it.  The device bins
 * min(total, capacity) records (read back by svr_binning_count) and sets status bit 8 when
 * records were dropped; path_or may be the OR over all voxel paths (a superset; status bit
 * 16 flags a path with bits the trimmed key would drop).  svr_workspace_query returns the
 * geom, binning and image buffer sizes {sizes[0], sizes[1], sizes[2]} for a capacity. */
SVR_API int svr_binning_count(const void* binning_buffer, int64_t* count_host, void* stream);
/* Candidate rows (no counterpart in the reference): the CTA-wide forward (svr_render_set_impl 3,
 * the default) stores, for every slot of 128 records it streams, each pixel's 128-bit mask of
 * the records whose box its ray meets; the CTA-wide adjoint then reads these rows, limited to
 * each pixel's last contributor, instead of testing the records again (the same masks, so the
 * same gradients).  The rows are valid after such a forward and until the next binning or a
 * forward of another kernel family (those repack the records without rows); otherwise the
 * adjoint filters as before.  svr_binning_candidates_valid reads that state (synchronises). */
SVR_API int svr_binning_candidates_valid(const void* binning_buffer, int* valid_host, void* stream);

/* Dense ranks (no counterpart in the reference): svr_rank_table_build sorts the trimmed rank
 * (octpath ^ octant pattern, low groups dropped as for path_or) of every (voxel, octant) pair
 * once per octree and writes table u32[8N] (index voxel * 8 + octant) = the pair's index
 * among the distinct ranks, and *rank_bits_host = the bits that index needs (synchronises;
 * workspace from svr_rank_table_workspace_bytes).  svr_bin_and_sort_ranked is
 * svr_bin_and_sort with the table's index in place of the rank in the sort key: the same
 * order and ties (the index orders as the rank does), a key narrower by up to
 * 3 * levels - rank_bits bits, so fewer radix passes.  path_or must be the one the table was
 * built with (it sets the trimming). */
SVR_API int svr_rank_table_workspace_bytes(int64_t N, size_t* bytes);
SVR_API int svr_rank_table_build(int64_t N, const int64_t* octpaths, uint64_t path_or, uint32_t* table,
                                 int* rank_bits_host, void* ws, size_t ws_bytes, void* stream);
SVR_API int svr_bin_and_sort_ranked(const svr_view_t* views_host, int n_views, int N, int64_t num_rendered,
                                    uint64_t path_or, const int64_t* octpaths, const uint32_t* rank_table,
                                    int rank_table_bits, void* geom_buffer, void* binning_buffer,
                                    size_t binning_bytes, void* image_buffer, void* stream);
SVR_API int svr_workspace_query(int n_views, int N, int64_t capacity, int64_t total_pixels,
                                int total_tiles, size_t* sizes_host);

/* Sorted per-tile values (octant << 29 | voxel id) and tile ranges, for tests. */
SVR_API int svr_unpack_binning(const void* binning_buffer, int64_t num_rendered, int total_tiles,
                       const void* image_buffer, int64_t total_pixels, uint32_t* vals,
                       uint32_t* ranges, uint32_t* tile_last, uint32_t* n_contrib, void* stream);

/* ---------------------------------------------------------------- render
 * Replaces _C.rasterize_voxels (cuda/src/forward.cu:986-1096) for the SDF density mode.
 * geos f32[N,8], rgbs f32[n_rgb_views*N, 3] (one block per view when n_rgb_views ==
 * n_views, else shared), s_val f32[1] on the device.  Outputs are packed per view (see
 * svr_view_t): color f32[3*P], depth f32[4*P] (may be NULL when !need_depth), normal
 * f32[3*P] (NULL when !need_normal), T f32[P], max_w f32[N] (NULL unless tracking).
 * n_samp in {1,2,3} (vox_geo_mode triinterp1 / triinterp / triinterp3). */
SVR_API int svr_render_fwd(const svr_view_t* views_host, int n_views, int N, int64_t num_rendered,
                   int n_samp, int need_depth, int need_normal,
                   const float* centers, const float* lengths, const float* geos, const float* rgbs,
                   int n_rgb_views, const float* s_val, void* geom_buffer, void* binning_buffer,
                   void* image_buffer, float* out_color, float* out_depth, float* out_normal,
                   float* out_T, float* max_w, void* stream);

/* Replaces _C.rasterize_voxels_backward (cuda/src/backward.cu:986-1109), SDF density
 * (always three sub-samples, backward.cu:944-946).  Accumulates into dL_dvox f32[N,12]
 * ([8 corner SDF | 3 rgb | |dL/dalpha * alpha|], caller zeroes it; with n_rgb_views ==
 * n_views the rgb gradient goes to drgbs f32[n_views*N,3] instead when non-NULL) and
 * dL_ds f32[1].  gt_color f32[3*P] is read only when lambda_R_concen > 0. */
SVR_API int svr_render_bwd(const svr_view_t* views_host, int n_views, int N, int64_t num_rendered,
                   int need_depth, int need_normal, float lambda_R_concen, const float* gt_color,
                   const float* s_val, void* binning_buffer, void* image_buffer,
                   const float* out_T, const float* dL_dcolor, const float* dL_ddepth,
                   const float* dL_dnormal, const float* dL_dT,
                   float* dL_dvox, float* drgbs, float* dL_ds, void* stream);

/* Launch variants of the render kernels (no counterpart in the reference): kernel family (as
 * svr_render_set_impl numbers them), ring slots and CTAs per SM, which change the schedule
 * only (every variant gives the same forward outputs and the same gradients up to the order of
 * float atomics).  pass 0 = forward, 1 = adjoint.  Variant 0 is the family chosen by
 * svr_render_set_impl (default 3) in its default configuration (for family 0 it follows the
 * launch size); the others name their family.  svr_render_set_impl resets the choice to 0.
 * The choice is process-wide and read when a launch is issued; svraster_b200.autotune times
 * the variants on the caller's workload. */
SVR_API int svr_render_config_count(int* n_fwd, int* n_bwd);
SVR_API int svr_render_config_describe(int pass, int index, int* impl, int* ring, int* ctas_per_sm);
SVR_API int svr_render_set_config(int fwd_index, int bwd_index);
SVR_API int svr_render_get_config(int* fwd_index, int* bwd_index);

/* Forward with per-view max blending weights (compute_training_stat,
 * src/sparse_voxel_gears/adaptive.py:80-113, renders every view with track_max_w): as
 * svr_render_fwd, but max_w_views f32[n_views, N] (caller zeroes it) gets one row per view. */
SVR_API int svr_render_fwd_max_w_views(const svr_view_t* views_host, int n_views, int N,
                                       int64_t num_rendered, int n_samp, int need_depth,
                                       int need_normal, const float* centers, const float* lengths,
                                       const float* geos, const float* rgbs, int n_rgb_views,
                                       const float* s_val, void* geom_buffer, void* binning_buffer,
                                       void* image_buffer, float* out_color, float* out_depth,
                                       float* out_normal, float* out_T, float* max_w_views,
                                       void* stream);

/* Binning without a global radix sort (no counterpart in the reference; same result as
 * svr_bin_and_sort, whose order is the one of cuda/src/forward.cu:749-829, 882-939).
 * svr_pair_order_build (once per octree): pair_pos u32[8N], octant-major (entry q*N + v) = the
 * position of the pair (voxel v, octant q) in the order of the full octree rank, ties by voxel
 * id then octant;
 * *key_bits_host = bits of a position.  The workspace is svr_rank_table_workspace_bytes(N).
 * svr_bin_tiles (per step, after svr_preprocess): counts the records of every tile, scans
 * the counts into tile ranges and the heavy-first launch order, scatters every record into
 * its tile's range, and sorts each tile by pair position with one CTA.  R is the record
 * capacity (the device bins min(total, R) records and sets status bit 8 beyond it); no host
 * synchronisation, so it can be captured into a CUDA graph. */
/* Record total and path OR of a preprocessed batch (one 16-byte read and a stream
 * synchronisation, no scan): what svr_bin_tiles needs to size its buffers.  No counterpart in
 * the reference (its count is the scan's last entry, forward.cu:855-880). */
SVR_API int svr_rendered_total(const void* geom_buffer, int64_t* num_rendered_host, uint64_t* path_or_host,
                               void* stream);
SVR_API int svr_pair_order_build(int64_t N, const int64_t* octpaths, uint32_t* pair_pos, int* key_bits_host,
                                 void* ws, size_t ws_bytes, void* stream);
SVR_API int svr_bin_tiles(const svr_view_t* views_host, int n_views, int N, int64_t R, const uint32_t* pair_pos,
                          int key_bits, void* geom_buffer, void* binning_buffer, size_t binning_bytes,
                          void* image_buffer, void* stream);

/* Which render kernels later launches use (no counterpart in the reference; a process-wide
 * choice read when a launch is issued), for the forward and the adjoint: 0 = per-warp filter
 * with one pixel per lane, 1 = record-parallel filter with dense pair evaluation, warps on
 * 8x4 pixel blocks, 2 = the same with every warp on a lattice spread over the tile, 3 (the
 * default) = the same with a slot's pairs numbered and evaluated over the whole CTA.  Every choice gives the same forward outputs bit for bit and the same gradients up to
 * the order of their float atomics. */
SVR_API int svr_render_set_impl(int fwd_impl, int bwd_impl);
SVR_API int svr_render_get_impl(int* fwd_impl, int* bwd_impl);

/* Stage timing, no counterpart in the reference: a CUDA event (cudaEvent_t, or null for none)
 * that every later svr_render_fwd records on its stream between its record packing launch and
 * its render launch.  A process-wide setting; leave it null while a CUDA graph is captured. */
SVR_API int svr_set_pack_event(void* event);

/* Work measurement, no counterpart in the reference: the forward render of
 * svr_render_fwd (three sub-samples, depth and normal on) on records already packed by an
 * earlier svr_render_fwd on the same buffers, with the same outputs, that also writes to
 * pair_count (device u64[3]) the (pixel, record) pairs that reached the SDF evaluation, those
 * with alpha >= MIN_ALPHA, and those up to each pixel's last contributor (the pairs the adjoint
 * evaluates).  A separate kernel instance: the plain forward does not count. */
SVR_API int svr_render_fwd_count_pairs(const svr_view_t* views_host, int n_views, int N, int64_t R,
                                       const float* s_val, void* binning_buffer, void* image_buffer,
                                       float* out_color, float* out_depth, float* out_normal, float* out_T,
                                       unsigned long long* pair_count, void* stream);

/* Device status word of the raster launches that used this image buffer (0 = clean;
 * bit 1 wait timeout, bit 2 index out of range, bit 4 duplicate count mismatch, bit 8
 * records beyond the binning capacity, bit 16 sort-key format, bit 64 a render CTA that had
 * timed out exited while one of its bulk copies had not been seen to land: the launch's
 * outputs are undefined and the process should not trust the device afterwards).
 * Synchronises `stream`.  Replaces the reference's __trap() sanity checks
 * (preprocess.cu:141-146, forward.cu:796-801, backward.cu:126-137). */
SVR_API int svr_read_status(const void* image_buffer, int64_t total_pixels, int total_tiles,
                    uint32_t* status_host, void* stream);

/* ---------------------------------------------------------------- per-voxel parameters
 * Replace _C.gather_triinterp_geo_params[_bw] (cuda/src/geo_params_gather.cu:134-173). */
SVR_API int svr_gather_geo(int64_t n_care, const int64_t* care_idx, const int64_t* vox_key,
                   const float* grid_pts, float* geos, void* stream);
SVR_API int svr_gather_geo_bw(int64_t n_care, const int64_t* care_idx, const int64_t* vox_key,
                      const float* dL_dgeos, float* dL_dgrid, void* stream);

/* Scatter per-voxel corner gradients with row stride ld (8 for dL_dgeos, 12 for the render
 * adjoint's dL_dvox) into dL_dgrid f32[M] for all N voxels: the gather adjoint of
 * geo_params_gather.cu:48-72 applied directly to the render output (batched training step). */
SVR_API int svr_scatter_vox_grads(int64_t N, int ld, const int64_t* vox_key, const float* dvox,
                                  float* dL_dgrid, void* stream);

/* Replace _C.sh_compute / _C.sh_compute_bw (cuda/src/sh_compute.cu:243-299).  n_idx == 0
 * means all N voxels.  sh0 f32[N,3], shs f32[N,M-1,3]. */
SVR_API int svr_sh_eval(int N, int64_t n_idx, const int64_t* idx, int degree, int M,
                const float* centers, const float* cam_pos, const float* sh0, const float* shs,
                float* rgbs, void* stream);
SVR_API int svr_sh_eval_bw(int N, int64_t n_idx, const int64_t* idx, int degree, int M,
                   const float* centers, const float* cam_pos, const float* dL_drgbs,
                   float* dL_dsh0, float* dL_dshs, void* stream);

/* Multi-view SH for a batch of views (sh_compute.cu:55-176 per view): rgbs f32[V,N,3] for
 * camera positions cam_pos f32[V,3]; the adjoint sums every view's colour gradient
 * drgbs f32[V,N,3] into dL_dsh0 f32[N,3] / dL_dshs f32[N,M-1,3] (written, not accumulated). */
SVR_API int svr_sh_eval_views(int N, int n_views, int degree, int M, const float* centers,
                              const float* cam_pos, const float* sh0, const float* shs, float* rgbs,
                              void* stream);
SVR_API int svr_sh_eval_views_bw(int N, int n_views, int degree, int M, const float* centers,
                                 const float* cam_pos, const float* drgbs, float* dL_dsh0,
                                 float* dL_dshs, void* stream);
/* The same adjoint added to dL_dsh0 / dL_dshs (a step that renders its views in several
 * chunks sums every chunk's contribution); no counterpart in the reference. */
SVR_API int svr_sh_eval_views_bw_add(int N, int n_views, int degree, int M, const float* centers,
                                     const float* cam_pos, const float* drgbs, float* dL_dsh0,
                                     float* dL_dshs, void* stream);

/* ---------------------------------------------------------------- grid regularisers
 * Replace _C.valid_gradient_table (cuda/src/utils.cu:362-408) + the key sort of
 * src/utils/octree_utils.py:293-314.  Two calls sharing one workspace: count (synchronises;
 * workspace >= svr_valid_table_workspace_bytes(N, 0)), then fill (workspace >=
 * svr_valid_table_workspace_bytes(N, count)).  grid_mask is u8[res^3], res = 2^res_pow2. */
SVR_API size_t svr_valid_table_workspace_bytes(int N, int64_t count);
SVR_API int svr_valid_table_count(int N, const float* centers, const float* sizes,
                          const float* scene_center, float inside_extent, int res_pow2,
                          const uint8_t* is_leaf, void* workspace, int64_t* count_host,
                          void* stream);
SVR_API int svr_valid_table_fill(int N, const float* centers, const float* sizes,
                         const float* scene_center, float inside_extent, int res_pow2,
                         const uint8_t* is_leaf, int64_t count, void* workspace,
                         uint8_t* grid_mask, int32_t* grid_keys, int32_t* grid2voxel,
                         void* stream);

/* Direct-mapped index of the sorted grid keys: dense_index i32[grid_res^3] gets the table row
 * of every registered cell and -1 elsewhere.  Optional input of the smoothness adjoints (no
 * counterpart in the reference, which binary-searches the keys, auxiliary.h:418-427). */
SVR_API int svr_grid_index_build(int G, const int32_t* grid_keys, int grid_res,
                                 int32_t* dense_index, uint32_t* status, void* stream);

/* Replace _C.laplacian_smoothness_bw (cuda/src/ls_compute.cu:111-153) and
 * _C.grid_eikonal_bw (cuda/src/ge_compute.cu:119-160); accumulate into grid_grad f32[M].
 * `seed` replaces the reference's clock64() seed so runs are reproducible; `status` is a
 * device u32 that collects index errors (0 when clean).  dense_index (from
 * svr_grid_index_build) may be NULL, in which case keys are binary-searched. */
SVR_API int svr_laplacian_bw(int G, int A, const int32_t* active, const int32_t* grid_keys,
                     const int32_t* grid2voxel, int grid_res, const uint8_t* grid_mask,
                     const int32_t* dense_index, const float* voxel_coords, const float* voxel_sizes, int N,
                     const int64_t* vox_key, const float* grid_pts, int M, float weight,
                     float vox_size_inv, int seed, float* grid_grad, uint32_t* status,
                     void* stream);
SVR_API int svr_eikonal_bw(int G, int A, const int32_t* active, const int32_t* grid_keys,
                   const int32_t* grid2voxel, int grid_res, const uint8_t* grid_mask,
                   const int32_t* dense_index, const float* voxel_coords, const float* voxel_sizes, int N,
                   const int64_t* vox_key, const float* grid_pts, int M, float weight,
                   float vox_size_inv, int seed, float* grid_grad, uint32_t* status,
                   void* stream);

/* The other grid regularisers.  svr_voxel_gradient_bw replaces _C.voxel_gradient_bw
 * (cuda/src/vg_compute.cu:23-118) for the A voxels of active; svr_total_variation_bw replaces
 * _C.total_variation_bw (cuda/src/tv_compute.cu:23-176) for grid values f32[M,C]: with
 * tv_sparse the participating voxels are decided from grid_grad as it is on entry (the
 * reference reads it while adding to it), valid_ws u8[N*C] is scratch; svr_points_loss_bw
 * replaces _C.points_loss_bw (cuda/src/pl_compute.cu:14-108) for points f32[P,3] in grid
 * units, dense_index optional (svr_grid_index_build).  All add into grid_grad. */
SVR_API int svr_voxel_gradient_bw(int N, int A, const int32_t* active, const int64_t* vox_key,
                                  const float* grid_pts, int64_t M, const float* vox_size_inv,
                                  float weight, float* grid_grad, uint32_t* status, void* stream);
SVR_API int svr_total_variation_bw(int64_t N, int C, const int64_t* vox_key, const float* grid_pts,
                                   int64_t M, float weight, const float* vox_size_inv, int no_tv_s,
                                   int tv_sparse, uint8_t* valid_ws, float* grid_grad,
                                   uint32_t* status, void* stream);
SVR_API int svr_points_loss_bw(int P, const float* points_in_grid, int G, const int32_t* grid_keys,
                               const int32_t* grid2voxel, int grid_res, const uint8_t* grid_mask,
                               const int32_t* dense_index, const float* voxel_coords,
                               const float* voxel_sizes, int N, const int64_t* vox_key,
                               const float* grid_pts, int M, float weight, float* grid_grad,
                               uint32_t* status, void* stream);

/* Spatially ordered forms of svr_voxel_gradient_bw and svr_total_variation_bw (no
 * counterpart in the reference, whose kernels visit voxels in storage order,
 * vg_compute.cu:23-77, tv_compute.cu:22-158).  svr_voxel_order sorts the voxels once per
 * octree by the grid-point index of their first corner: order i32[N] (visit position ->
 * voxel, ties by voxel id) and rank i32[N] (its inverse); workspace from
 * svr_voxel_order_workspace_bytes.  The _ordered adjoints take that order and rank as
 * produced there (they are not range-checked); count_ws i32[N], valid_ws u8[N*C] are
 * scratch.  Same results as the storage-order forms up to the order of float additions.
 * vox_key 16-byte aligned. */
SVR_API int svr_voxel_order_workspace_bytes(int64_t N, size_t* bytes);
SVR_API int svr_voxel_order(int64_t N, const int64_t* vox_key, int64_t M, int32_t* order, int32_t* rank,
                            void* ws, size_t ws_bytes, uint32_t* status, void* stream);
SVR_API int svr_voxel_gradient_bw_ordered(int N, int A, const int32_t* active, const int32_t* order,
                                          const int32_t* rank, const int64_t* vox_key, const float* grid_pts,
                                          int64_t M, const float* vox_size_inv, float weight,
                                          int32_t* count_ws, float* grid_grad, uint32_t* status,
                                          void* stream);
SVR_API int svr_total_variation_bw_ordered(int64_t N, int C, const int32_t* order, const int64_t* vox_key,
                                           const float* grid_pts, int64_t M, float weight,
                                           const float* vox_size_inv, int no_tv_s, int tv_sparse,
                                           uint8_t* valid_ws, float* grid_grad, uint32_t* status,
                                           void* stream);

/* Graph-replayable forms (no counterpart in the reference): the jitter seed is
 * seed_base + *step, read from a device counter (svr_counter_add) when the kernel runs. */
SVR_API int svr_laplacian_bw_at_step(int G, int A, const int32_t* active, const int32_t* grid_keys,
                                     const int32_t* grid2voxel, int grid_res, const uint8_t* grid_mask,
                                     const int32_t* dense_index, const float* voxel_coords,
                                     const float* voxel_sizes, int N, const int64_t* vox_key,
                                     const float* grid_pts, int M, float weight, float vox_size_inv,
                                     int seed_base, const int64_t* step, float* grid_grad,
                                     uint32_t* status, void* stream);
SVR_API int svr_eikonal_bw_at_step(int G, int A, const int32_t* active, const int32_t* grid_keys,
                                   const int32_t* grid2voxel, int grid_res, const uint8_t* grid_mask,
                                   const int32_t* dense_index, const float* voxel_coords,
                                   const float* voxel_sizes, int N, const int64_t* vox_key,
                                   const float* grid_pts, int M, float weight, float vox_size_inv,
                                   int seed_base, const int64_t* step, float* grid_grad,
                                   uint32_t* status, void* stream);

/* Fused Laplacian + grid-Eikonal adjoint accumulated per voxel corner (no counterpart in
 * the reference; equal, up to the order of floating-point additions, to svr_laplacian_bw
 * with weight w_ls plus svr_eikonal_bw with weight w_ge, both with `seed`, followed by the
 * grid scatter of dvox): adds each sample's corner gradients to dvox[v*ld + 0..7] of its
 * owner voxel v, for svr_scatter_vox_grads to move to the grid points.  geos f32[N,8]
 * (16-byte aligned) must hold grid[vox_key] of the current grid (svr_gather_geo);
 * dense_index is required; active may be NULL for all G table rows in order (A <= G);
 * seed_step may be NULL, else the seed is seed + *seed_step read on the device.  A zero
 * weight skips that loss. */
SVR_API int svr_smoothness_bw_vox(int G, int A, const int32_t* active, const int32_t* grid_keys,
                                  const int32_t* grid2voxel, int grid_res, const uint8_t* grid_mask,
                                  const int32_t* dense_index, const float* voxel_coords,
                                  const float* voxel_sizes, int N, const float* geos, float w_ls,
                                  float w_ge, float vox_size_inv, int seed, const int64_t* seed_step,
                                  float* dvox, int ld, uint32_t* status, void* stream);

/* Allocation-free variant of svr_laplacian_bw, for callers that cannot allocate device
 * memory (a host that reserves all device memory in a fixed arena at start-up and forbids
 * later cudaMalloc calls).  It has no counterpart in the reference.  The direct-mapped key
 * index lives in a static 8 MiB device array inside the library instead of caller memory,
 * so grid_res must be at most 128 (larger grids return SVR_ERR_CAPACITY; grid_res <= 0 is
 * SVR_ERR_ARG).  Inputs, outputs and the status word are the caller's, as for
 * svr_laplacian_bw, and no device memory is allocated.  The first call on each device
 * resolves the array's device address (cudaGetSymbolAddress); make that first call before
 * any stream capture.  The address is cached per device and context: after cudaDeviceReset
 * the next call resolves it again.  All calls share the one array and rebuild it each time,
 * so calls that overlap on the GPU race. */
SVR_API int svr_laplacian_bw_noalloc(int G, int A, const int32_t* active, const int32_t* grid_keys,
                                     const int32_t* grid2voxel, int grid_res, const uint8_t* grid_mask,
                                     const float* voxel_coords, const float* voxel_sizes, int N,
                                     const int64_t* vox_key, const float* grid_pts, int M, float weight,
                                     float vox_size_inv, int seed, float* grid_grad, uint32_t* status,
                                     void* stream);

/* ---------------------------------------------------------------- surface extraction
 * TSDF fusion, replacing src/utils/fuser_utils.py:54-156 (Fuser.integrate / tsdf): fold a batch
 * of views into the running weight / weighted-SDF sums of M grid points xyz f32[M,3].
 * Depth (and optional alpha) maps are packed per view like the render outputs: view v's
 * plane `sel` of a `ch`-channel image starts at ch * pix_offset_v + sel * H_v * W_v
 * (pix_offset is recomputed from the view sizes).  alpha_is_T reads alpha as 1 - T.
 * proj_host (may be NULL) holds per view the double tanfovx, tanfovy, cx/W, cy/H of the
 * camera (src/cameras.py:89-103).  Per-point 1/trunc (inv_trunc_pts) overrides `trunc`.
 * fp64 != 0: accumulators are f64, else f32 (the reference's order of rounding). */
SVR_API int svr_tsdf_integrate(const svr_view_t* views_host, const double* proj_host, int n_views,
                               int64_t M, const float* xyz, const float* depth, int depth_ch,
                               int depth_sel, const float* alpha, int alpha_ch, int alpha_sel,
                               int alpha_is_T, const float* inv_trunc_pts, double trunc,
                               double crop_border, float alpha_thres, int use_trunc,
                               int depth_weight, int border_weight, float max_norm_dist, int fp64,
                               void* weight_acc, void* sdf_acc, void* stream);

/* Sparse marching cubes, replacing cuda/svraster_cuda/marching_cubes.py:278-380
 * (torch_marching_cubes_grid): voxels vox_key i64[n_vox,8] over grid values f32[M] and
 * positions f32[M,3].  svr_mc_count classifies the voxels and returns the triangle count
 * (synchronises); svr_mc_emit writes the unique vertices (lexicographically sorted, as
 * unique(dim=0) returns them) into verts f32[>=3*n_tri,3] and faces i64[n_tri,3], and returns
 * the vertex count.  Both use one workspace: >= svr_mc_workspace_bytes(n_vox, 0) for the
 * count and >= svr_mc_workspace_bytes(n_vox, n_tri) for the emit, whose prefix must hold the
 * count's results.  fp64 interpolates the vertices in double (precision mode). */
SVR_API size_t svr_mc_workspace_bytes(int64_t n_vox, int64_t n_tri);
SVR_API int svr_mc_count(int64_t n_vox, const int64_t* vox_key, int64_t M, const float* grid_val,
                         float iso, void* workspace, int64_t* n_tri_host, void* stream);
SVR_API int svr_mc_emit(int64_t n_vox, const int64_t* vox_key, const float* grid_val,
                        const float* grid_xyz, float iso, int64_t n_tri, int fp64, void* workspace,
                        float* verts, int64_t* faces, int64_t* n_verts_host, void* stream);

/* ---------------------------------------------------------------- adaptive pruning / subdivision
 * svr_grid_link replaces octree_utils.build_grid_pts_link (src/utils/octree_utils.py:203-222):
 * for N voxels (octpath i64[N], octlevel i8[N]) writes the M unique corner grid points
 * grid_pts_key i64[M,3] (finest-level integer coordinates, lexicographic order as
 * unique(dim=0); capacity 8N rows) and vox_key i64[N,8] (their indices), returns M
 * (synchronises).  svr_subdivide_interp replaces adaptive.subdivide_by_interp
 * (adaptive.py:374-411): vox_val f32[n,8,C] -> out f32[8n,8,C].  svr_agg_voxel_into_grid_pts
 * replaces adaptive.agg_voxel_into_grid_pts (adaptive.py:349-372, index_reduce_ mean with
 * include_self=False): out f32[M,C], count_ws f32[M] scratch.  svr_training_stat_reduce
 * finishes compute_training_stat (adaptive.py:80-113) from per-view max weights
 * f32[n_views,N]: max_w, min_samp_interval and view_cnt f32[N] (initialised by the caller to
 * 0, 1e30 and 0) are updated in place; per view cam_pos / cam_lookat f32[3] and pix_size. */
SVR_API size_t svr_grid_link_workspace_bytes(int64_t N);
SVR_API int svr_grid_link(int64_t N, const int64_t* octpath, const int8_t* octlevel, void* workspace,
                          size_t workspace_bytes, int64_t* grid_pts_key, int64_t* vox_key,
                          int64_t* M_host, uint32_t* status, void* stream);
SVR_API int svr_subdivide_interp(int64_t n, int C, const float* vox_val, float* out, void* stream);
SVR_API int svr_agg_voxel_into_grid_pts(int64_t N, int C, const int64_t* vox_key, const float* vox_val,
                                        int64_t M, float* out, float* count_ws, uint32_t* status,
                                        void* stream);
SVR_API int svr_training_stat_reduce(int n_views, int64_t N, const float* max_w_views,
                                     const float* centers, const float* cam_pos,
                                     const float* cam_lookat, const float* pix_size, float* max_w,
                                     float* min_samp_interval, float* view_cnt, void* stream);

/* ---------------------------------------------------------------- normal-from-depth losses
 * svr_normal_depth_loss replaces the torch losses NormalDepthConsistencyLoss (mode 0,
 * src/utils/loss_utils.py:345-379: depth plane 0, alpha = 1 - T weighting, tolerance mask
 * tol_cos > 0) and NormalMedianConsistencyLoss (mode 1, loss_utils.py:381-407: depth plane
 * 2; tol_cos ignored) with cameras.py:104-127 (depth2pts / depth2normal, ks odd <= 9), for
 * all views in one launch.  depth f32[4*P], normal f32[3*P], T f32[P] packed per view as the
 * render outputs; loss_out f64[n_views] += weight * loss of each view; the gradient of that
 * is ADDED into grad_depth (the used plane) and grad_normal, the upstream planes of
 * svr_render_bwd. */
SVR_API int svr_normal_depth_loss(const svr_view_t* views_host, int n_views, int mode, int ks,
                                  float tol_cos, float weight, const float* depth, const float* normal,
                                  const float* T, double* loss_out, float* grad_depth,
                                  float* grad_normal, void* stream);

/* ---------------------------------------------------------------- checkpoint codebook
 * svr_quantize replaces io.quantization (src/sparse_voxel_gears/io.py:123-167, torch in the
 * reference): the 8-bit codebook of a quantized checkpoint for n float32 values (1 <= n <
 * 2^31): index_out u8[n], codebook_out f32[256]; workspace from svr_quantize_workspace_bytes.
 * Synchronises `stream` once per round (the rounds stop when nothing moves); *rounds_host
 * (may be NULL) gets the number of rounds that moved values; status bit 32 flags a
 * non-finite value.  Means are summed in float64, the reference's in float32.
 * svr_dequantize replaces io.dequantization (io.py:169-170): out f32[n] = codebook[index]. */
SVR_API int svr_quantize_workspace_bytes(int64_t n, size_t* bytes);
SVR_API int svr_quantize(int64_t n, const float* values, int max_iter, uint8_t* index_out,
                         float* codebook_out, void* ws, size_t ws_bytes, int* rounds_host,
                         uint32_t* status, void* stream);
SVR_API int svr_dequantize(int64_t n, const uint8_t* index, const float* codebook, float* out,
                           void* stream);

/* ---------------------------------------------------------------- optimiser
 * Replace _C.unbiased_adam_step / _C.biased_adam_step (cuda/src/adam_step.cu:106-159). */
SVR_API int svr_adam_step(int64_t numel, int biased, int sparse, float* param, const float* grad,
                  float* exp_avg, float* exp_avg_sq, double step, double lr, double beta1,
                  double beta2, float eps, void* stream);

/* BF16 storage of SH coefficients (no counterpart in the reference; the precision
 * configuration): svr_sh_eval_views_bf16 reads sh0 / shs as bf16 triples (converted exactly to
 * f32; all arithmetic f32) and writes f32 colours like svr_sh_eval_views.  The adjoint stays
 * svr_sh_eval_views_bw with f32 gradients.  svr_adam_step_bf16[_at] update bf16 parameters
 * with f32 moments: the step is computed in f32 from the stored value and rounded to nearest
 * bf16. */
SVR_API int svr_sh_eval_views_bf16(int N, int n_views, int degree, int M, const float* centers,
                                   const float* cam_pos, const uint16_t* sh0, const uint16_t* shs,
                                   float* rgbs, void* stream);
SVR_API int svr_adam_step_bf16(int64_t numel, int biased, int sparse, uint16_t* param, const float* grad,
                               float* exp_avg, float* exp_avg_sq, double step, double lr, double beta1,
                               double beta2, float eps, void* stream);
SVR_API int svr_adam_step_bf16_at(int64_t numel, int biased, int sparse, uint16_t* param,
                                  const float* grad, float* exp_avg, float* exp_avg_sq,
                                  const float* coef_table, int64_t rows, const int64_t* step,
                                  double beta1, double beta2, float eps, uint32_t* status,
                                  void* stream);

/* Graph-replayable Adam (no counterpart in the reference): the step number is read from a
 * device counter when the kernel runs and indexes a table of per-step coefficients
 * {lr / (1 - beta1^t), 1 / sqrt(1 - beta2^t)} that svr_adam_coef_table fills on the host
 * in double, exactly as svr_adam_step computes them.  A step outside [1, rows) sets bit 2
 * of `status` and leaves the parameters unchanged.  svr_counter_add adds `delta` to a
 * device int64 counter in stream order. */
SVR_API int svr_adam_coef_table(int biased, double lr, double beta1, double beta2, int64_t rows,
                                float* table_host);
SVR_API int svr_adam_step_at(int64_t numel, int biased, int sparse, float* param, const float* grad,
                             float* exp_avg, float* exp_avg_sq, const float* coef_table, int64_t rows,
                             const int64_t* step, double beta1, double beta2, float eps,
                             uint32_t* status, void* stream);
SVR_API int svr_counter_add(int64_t* counter, int64_t delta, void* stream);

/* ---------------------------------------------------------------- batched training step
 * The whole multi-view training step as one native object, for hosts that are not Python (no
 * counterpart in the reference, which steps one view at a time from Python, train.py:324-709).
 * One step: corner-SDF gather, SH colour of every view, preprocess, per-tile binning, render
 * forward (three sub-samples, depth and normal), render adjoint, the fused Laplacian +
 * grid-Eikonal adjoint (train.py:540-620), the corner-gradient scatter to the grid points, the
 * SH adjoint, and Adam (unbiased, dense) on grid, sh0 and shs.  The upstream gradients
 * dL/d(colour, depth, normal, T) (the photometric and normal-consistency losses run upstream of
 * the rasterizer) are planes the step owns and the caller fills before each step.
 *
 * The caller owns the octree and the parameters (device memory that must outlive the step; Adam
 * updates grid, sh0 and shs in place).  The step owns everything else, allocated once by
 * svr_step_create: the record buffers (sized for the record count of the views, found by one
 * counting pass, or for desc.record_capacity), the dense grid tables of the smoothness losses
 * (built from the octree), Adam's moments and per-step coefficient table, and the output and
 * upstream planes.  The views' matrices and backgrounds are copied, so the caller's may go.
 * svr_step_create synchronises `stream`; a new octree or new views need a new step object. */
typedef struct svr_step svr_step_t;

typedef struct {
    /* octree (device): N voxels */
    int32_t n_vox;
    int32_t sh_degree;              /* 0..3; sh0 f32/bf16[N,3], shs f32/bf16[N, (deg+1)^2 - 1, 3] */
    int32_t sh_bf16;                /* 1: sh0 / shs hold bf16 (uint16) values, moments stay f32 */
    int32_t grid_res_pow2;          /* dense grid of the smoothness losses: 2^p cells per side,
                                       p in 1..10 (train.py:599 uses the finest voxel level) */
    const int64_t* octpath;         /* [N] */
    const float* centers;           /* [N,3] */
    const float* lengths;           /* [N] */
    const uint8_t* is_leaf;         /* [N] */
    const int64_t* vox_key;         /* [N,8] grid point of each voxel corner */
    /* parameters (device, updated in place) */
    float* grid;                    /* [n_grid] corner SDF values */
    void* sh0;
    void* shs;
    int64_t n_grid;
    const float* s_val;             /* [1] SDF scale, read by the render kernels */
    /* scene box of the dense grid (train.py:180-181) */
    float scene_center[3];
    float inside_extent;
    /* losses and optimiser */
    float lambda_ls, lambda_ge;     /* Laplacian / grid-Eikonal weights (0 skips one) */
    float lambda_R_concen;          /* colour-concentration weight; >0 reads the SVR_STEP_GT plane */
    double lr[3];                   /* grid, sh0, shs */
    double beta1, beta2;
    float eps;
    int32_t seed;                   /* smoothness sampling seed; step t uses seed + t */
    int32_t adam_rows;              /* steps the coefficient table covers (0: 2^20) */
    int64_t record_capacity;        /* 0: the views' record count (counted at create) */
} svr_step_desc_t;

/* Buffers of a step object, for svr_step_buffer. */
typedef enum {
    SVR_STEP_COLOR = 0,     /* f32[3P] rendered colour (planar per view, as svr_render_fwd) */
    SVR_STEP_DEPTH = 1,     /* f32[4P] */
    SVR_STEP_NORMAL = 2,    /* f32[3P] */
    SVR_STEP_T = 3,         /* f32[P] transmittance */
    SVR_STEP_DCOLOR = 4,    /* f32[3P] upstream dL/dcolor (caller writes) */
    SVR_STEP_DDEPTH = 5,    /* f32[4P] upstream dL/ddepth (caller writes) */
    SVR_STEP_DNORMAL = 6,   /* f32[3P] upstream dL/dnormal (caller writes) */
    SVR_STEP_DT = 7,        /* f32[P] upstream dL/dT (caller writes; zero at create) */
    SVR_STEP_GT = 8,        /* f32[3P] ground-truth colour (only when lambda_R_concen > 0) */
    SVR_STEP_GRAD_FLAT = 9, /* f32 all parameter gradients, one contiguous buffer (the one a
                               data-parallel host all-reduces between the two phases) */
    SVR_STEP_GRAD_GRID = 10,/* f32[n_grid], a 256-byte aligned view into GRAD_FLAT */
    SVR_STEP_GRAD_SH0 = 11, /* f32[N*3] */
    SVR_STEP_GRAD_SHS = 12, /* f32[N*(M-1)*3] */
    SVR_STEP_DVOX = 13,     /* f32[N*12] per-voxel adjoint [8 corners | rgb | |dL/dalpha*alpha|] */
    SVR_STEP_DS = 14,       /* f32[1] dL/ds */
    SVR_STEP_STEP = 15,     /* int64[1] Adam steps taken (device counter) */
    SVR_STEP_N_BUFFERS = 16
} svr_step_buffer_t;

/* Phases of svr_step_run: 1 = everything up to the gradients in GRAD_FLAT, 2 = Adam (and the
 * step counter); 3 = both.  A data-parallel host runs 1, all-reduces GRAD_FLAT, runs 2. */
#define SVR_STEP_GRADS 1
#define SVR_STEP_ADAM 2

SVR_API int svr_step_create(const svr_step_desc_t* desc, const svr_view_t* views_host, int n_views,
                            void* stream, svr_step_t** out_host);
/* Waits for the device (the step's work may still be queued on the caller's streams), then
 * frees everything the step owns. */
SVR_API int svr_step_destroy(svr_step_t* step);
/* Device pointer and element count of one buffer (svr_step_buffer_t). */
SVR_API int svr_step_buffer(const svr_step_t* step, int which, void** ptr_host, int64_t* count_host);
/* info_host[0..7] = total pixels P, record capacity, total tiles, dense-grid table rows G,
 * GRAD_FLAT elements, views, kernels per step (phases 1+2), whether graphs are captured. */
SVR_API int svr_step_info(const svr_step_t* step, int64_t* info_host);
/* Run phases of one step on `stream` (asynchronous; after svr_step_capture by graph launch). */
SVR_API int svr_step_run(svr_step_t* step, int phases, void* stream);
/* Capture each phase into a CUDA graph, recorded on a stream of the step's own, so that any
 * stream, the legacy default included, may be passed; later svr_step_run calls launch the
 * graphs on their stream.  Runs phase 1 once eagerly on `stream` first (kernel attributes are
 * set outside the capture); parameters and the step counter are left as they were.
 * Synchronises `stream`. */
SVR_API int svr_step_capture(svr_step_t* step, void* stream);
/* Status words: the raster launches' (svr_read_status bits) and the smoothness / Adam kernels'
 * (bit 2: an index out of range or a step outside the coefficient table).  The second word
 * keeps its bits for the life of the step object.  Synchronises. */
SVR_API int svr_step_status(const svr_step_t* step, uint32_t* raster_host, uint32_t* other_host,
                            void* stream);

#ifdef __cplusplus
}
#endif
#endif
