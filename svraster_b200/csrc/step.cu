// The batched multi-view training step as one native object (svr_step_*).
//
// A host that is not Python drives the whole step through the C ABI: svr_step_create sizes and
// allocates every buffer once (records, dense smoothness grid, Adam state, output and upstream
// planes), svr_step_run issues the step's launches in order on one stream, and
// svr_step_capture records each phase into a CUDA graph on a stream of the step's own, so that
// later runs are two graph launches.  The launches are the library's own entry points, in the
// order the Python step (svraster_b200/step.py) issues them; the per-view reference sequence
// it replaces is train.py:324-709 (render, regularisers, optimiser step).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/svraster_b200.h"

int svr_fail(int code, const char* what);
void svr_note_launch(int n);

#define STEP_CUDA(x)                                                                          \
    do {                                                                                      \
        cudaError_t e_ = (x);                                                                 \
        if (e_ != cudaSuccess)                                                                \
            return svr_fail(SVR_ERR_CUDA, (std::string("step: ") + #x + ": " + cudaGetErrorString(e_)).c_str()); \
    } while (0)
#define STEP_TRY(x)                                                                           \
    do {                                                                                      \
        int r_ = (x);                                                                         \
        if (r_ != SVR_OK) return r_;                                                          \
    } while (0)

namespace {

constexpr int kPlaneColor = 0, kPlaneDepth = 1, kPlaneNormal = 2, kPlaneT = 3;
constexpr int kPlaneDColor = 4, kPlaneDDepth = 5, kPlaneDNormal = 6, kPlaneDT = 7, kPlaneGT = 8;
constexpr int kPlanes = 9;
constexpr int kPlaneWidth[kPlanes] = {3, 4, 3, 1, 3, 4, 3, 1, 3};   // floats per pixel

__global__ void iota64_kernel(int64_t n, int64_t* __restrict__ out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = i;
}

// Voxel origin and edge in dense-grid cells (train.py:180-181), rounded to the nearest cell
// (ties to even): ((c - l/2) - (centre - extent/2)) / extent * res, every operation rounded as
// float32.  With the scene centred at the origin this equals (c - l/2) + extent/2 bit for bit.
__global__ void grid_coords_kernel(int n, const float* __restrict__ centers, const float* __restrict__ lengths,
                                   float3 scene_center, float extent, float res, float* __restrict__ coords,
                                   float* __restrict__ sizes)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float l = lengths[i];
    const float half = __fmul_rn(l, 0.5f);
    const float half_ext = __fmul_rn(extent, 0.5f);
    const float c0[3] = {scene_center.x, scene_center.y, scene_center.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float lo = __fsub_rn(centers[3 * i + k], half);
        const float base = __fsub_rn(c0[k], half_ext);
        coords[3 * i + k] = rintf(__fmul_rn(__fdiv_rn(__fsub_rn(lo, base), extent), res));
    }
    sizes[i] = rintf(__fmul_rn(__fdiv_rn(l, extent), res));
}

inline int64_t round_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

}  // namespace

struct svr_step {
    svr_step_desc_t d{};
    int V = 0, N = 0, M_sh = 1, tiles = 0;
    int64_t P = 0, capacity = 0;
    std::vector<svr_view_t> views;
    std::vector<void*> allocs;
    // step-owned copies of the cameras: per view w2c[16] | c2w[16] | bg[4]; camera positions
    float* mats = nullptr;
    float* cam_pos = nullptr;
    float* scene_center = nullptr;
    // dense grid of the smoothness losses
    int G = 0, res = 0;
    float vox_size_min_inv = 0.f;
    uint8_t* grid_mask = nullptr;
    int32_t* grid_keys = nullptr;
    int32_t* grid2voxel = nullptr;
    int32_t* grid_index = nullptr;
    float* vcoord = nullptr;
    float* vsize = nullptr;
    // binning
    uint32_t* pair_pos = nullptr;
    int key_bits = 0;
    int64_t* all_idx = nullptr;
    int32_t* n_dup = nullptr;
    void* geom = nullptr;
    void* binning = nullptr;
    void* image = nullptr;
    size_t bin_bytes = 0;
    // per-step state
    float* geos = nullptr;
    float* rgbs = nullptr;
    float* drgbs = nullptr;
    float* dvox = nullptr;
    float* ds = nullptr;
    float* plane[kPlanes] = {};
    float* grad_flat = nullptr;
    int64_t n_flat = 0;
    float* grad[3] = {};
    int64_t numel[3] = {};
    float* adam_m[3] = {};
    float* adam_v[3] = {};
    float* coef[3] = {};
    int64_t rows = 0;
    int64_t* step_dev = nullptr;
    uint32_t* status = nullptr;
    // graphs
    cudaStream_t cap = nullptr;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    long long kernels[2] = {0, 0};

    template <typename T>
    int alloc(T** p, int64_t count)
    {
        void* q = nullptr;
        const size_t bytes = (size_t)std::max<int64_t>(count, 1) * sizeof(T);
        STEP_CUDA(cudaMalloc(&q, bytes));
        allocs.push_back(q);
        *p = static_cast<T*>(q);
        return SVR_OK;
    }
};

static int phase_grads(svr_step* h, cudaStream_t st)
{
    const svr_step_desc_t& d = h->d;
    const int N = h->N, V = h->V;
    void* s = (void*)st;
    STEP_TRY(svr_gather_geo(N, h->all_idx, d.vox_key, d.grid, h->geos, s));
    if (d.sh_bf16)
        STEP_TRY(svr_sh_eval_views_bf16(N, V, d.sh_degree, h->M_sh, d.centers, h->cam_pos, (const uint16_t*)d.sh0,
                                        (const uint16_t*)d.shs, h->rgbs, s));
    else
        STEP_TRY(svr_sh_eval_views(N, V, d.sh_degree, h->M_sh, d.centers, h->cam_pos, (const float*)d.sh0,
                                   (const float*)d.shs, h->rgbs, s));
    STEP_TRY(svr_preprocess(h->views.data(), V, N, d.centers, d.lengths, d.is_leaf, d.octpath, h->n_dup, h->geom, s));
    STEP_TRY(svr_bin_tiles(h->views.data(), V, N, h->capacity, h->pair_pos, h->key_bits, h->geom, h->binning,
                           h->bin_bytes, h->image, s));
    STEP_TRY(svr_render_fwd(h->views.data(), V, N, h->capacity, 3, 1, 1, d.centers, d.lengths, h->geos, h->rgbs, V,
                            d.s_val, h->geom, h->binning, h->image, h->plane[kPlaneColor], h->plane[kPlaneDepth],
                            h->plane[kPlaneNormal], h->plane[kPlaneT], nullptr, s));
    STEP_CUDA(cudaMemsetAsync(h->dvox, 0, (size_t)N * 12 * sizeof(float), st));
    STEP_CUDA(cudaMemsetAsync(h->drgbs, 0, (size_t)V * N * 3 * sizeof(float), st));
    STEP_CUDA(cudaMemsetAsync(h->ds, 0, sizeof(float), st));
    STEP_TRY(svr_render_bwd(h->views.data(), V, N, h->capacity, 1, 1, d.lambda_R_concen,
                            d.lambda_R_concen > 0.f ? h->plane[kPlaneGT] : nullptr, d.s_val, h->binning, h->image,
                            h->plane[kPlaneT], h->plane[kPlaneDColor], h->plane[kPlaneDDepth],
                            h->plane[kPlaneDNormal], h->plane[kPlaneDT], h->dvox, h->drgbs, h->ds, s));
    if (h->G > 0)
        STEP_TRY(svr_smoothness_bw_vox(h->G, h->G, nullptr, h->grid_keys, h->grid2voxel, h->res, h->grid_mask,
                                       h->grid_index, h->vcoord, h->vsize, N, h->geos, d.lambda_ls, d.lambda_ge,
                                       h->vox_size_min_inv, d.seed, h->step_dev, h->dvox, 12, h->status, s));
    STEP_CUDA(cudaMemsetAsync(h->grad_flat, 0, (size_t)h->n_flat * sizeof(float), st));
    STEP_TRY(svr_scatter_vox_grads(N, 12, d.vox_key, h->dvox, h->grad[0], s));
    STEP_TRY(svr_sh_eval_views_bw(N, V, d.sh_degree, h->M_sh, d.centers, h->cam_pos, h->drgbs, h->grad[1],
                                  h->grad[2], s));
    return SVR_OK;
}

static int phase_adam(svr_step* h, cudaStream_t st)
{
    const svr_step_desc_t& d = h->d;
    void* s = (void*)st;
    STEP_TRY(svr_counter_add(h->step_dev, 1, s));
    void* params[3] = {d.grid, d.sh0, d.shs};
    for (int k = 0; k < 3; ++k) {
        if (h->numel[k] == 0) continue;
        if (k > 0 && d.sh_bf16)
            STEP_TRY(svr_adam_step_bf16_at(h->numel[k], 0, 0, (uint16_t*)params[k], h->grad[k], h->adam_m[k],
                                           h->adam_v[k], h->coef[k], h->rows, h->step_dev, d.beta1, d.beta2, d.eps,
                                           h->status, s));
        else
            STEP_TRY(svr_adam_step_at(h->numel[k], 0, 0, (float*)params[k], h->grad[k], h->adam_m[k], h->adam_v[k],
                                      h->coef[k], h->rows, h->step_dev, d.beta1, d.beta2, d.eps, h->status, s));
    }
    return SVR_OK;
}

static int run_phase(svr_step* h, int phase, cudaStream_t st)
{
    const long long n0 = svr_kernel_launches();
    const int rc = phase == 0 ? phase_grads(h, st) : phase_adam(h, st);
    if (rc == SVR_OK) h->kernels[phase] = svr_kernel_launches() - n0;
    return rc;
}

// ------------------------------------------------------------------ create / destroy
static int check_desc(const svr_step_desc_t* d, const svr_view_t* views, int n_views)
{
    if (!d || !views) return svr_fail(SVR_ERR_ARG, "step: null descriptor or views");
    if (n_views <= 0 || n_views > SVR_MAX_VIEWS) return svr_fail(SVR_ERR_ARG, "step: view count out of 1..SVR_MAX_VIEWS");
    if (d->n_vox <= 0 || 8ll * d->n_vox >= (1ll << 29)) return svr_fail(SVR_ERR_ARG, "step: voxel count out of range");
    if (d->sh_degree < 0 || d->sh_degree > 3) return svr_fail(SVR_ERR_ARG, "step: sh_degree must be 0..3");
    if (d->grid_res_pow2 < 1 || d->grid_res_pow2 > 10) return svr_fail(SVR_ERR_ARG, "step: grid_res_pow2 must be 1..10");
    if (!(d->inside_extent > 0.f)) return svr_fail(SVR_ERR_ARG, "step: inside_extent must be positive");
    if (d->n_grid <= 0) return svr_fail(SVR_ERR_ARG, "step: n_grid must be positive");
    if (!d->octpath || !d->centers || !d->lengths || !d->is_leaf || !d->vox_key || !d->grid || !d->sh0 || !d->s_val ||
        (d->sh_degree > 0 && !d->shs))
        return svr_fail(SVR_ERR_ARG, "step: null octree or parameter pointer");
    if (d->adam_rows < 0 || d->record_capacity < 0) return svr_fail(SVR_ERR_ARG, "step: negative size");
    for (int v = 0; v < n_views; ++v)
        if (views[v].width <= 0 || views[v].height <= 0 || !views[v].w2c || !views[v].c2w)
            return svr_fail(SVR_ERR_ARG, "step: view without size or matrices");
    return SVR_OK;
}

static int build(svr_step* h, const svr_view_t* views_in, cudaStream_t st)
{
    const svr_step_desc_t& d = h->d;
    const int V = h->V, N = h->N;
    void* s = (void*)st;
    h->M_sh = (d.sh_degree + 1) * (d.sh_degree + 1);

    // cameras: the caller's matrices copied into one step-owned block
    std::vector<float> host((size_t)V * 36, 0.f);
    for (int v = 0; v < V; ++v) {
        float* m = &host[(size_t)v * 36];
        STEP_CUDA(cudaMemcpyAsync(m, views_in[v].w2c, 16 * sizeof(float), cudaMemcpyDeviceToHost, st));
        STEP_CUDA(cudaMemcpyAsync(m + 16, views_in[v].c2w, 16 * sizeof(float), cudaMemcpyDeviceToHost, st));
        if (views_in[v].bg)
            STEP_CUDA(cudaMemcpyAsync(m + 32, views_in[v].bg, 3 * sizeof(float), cudaMemcpyDeviceToHost, st));
    }
    STEP_CUDA(cudaStreamSynchronize(st));
    std::vector<float> cam((size_t)V * 3);
    for (int v = 0; v < V; ++v) {
        const float* c2w = &host[(size_t)v * 36 + 16];
        cam[3 * v] = c2w[3]; cam[3 * v + 1] = c2w[7]; cam[3 * v + 2] = c2w[11];
    }
    STEP_TRY(h->alloc(&h->mats, (int64_t)V * 36));
    STEP_TRY(h->alloc(&h->cam_pos, (int64_t)V * 3));
    STEP_TRY(h->alloc(&h->scene_center, 4));
    const float sc[4] = {d.scene_center[0], d.scene_center[1], d.scene_center[2], 0.f};
    STEP_CUDA(cudaMemcpyAsync(h->mats, host.data(), host.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    STEP_CUDA(cudaMemcpyAsync(h->cam_pos, cam.data(), cam.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    STEP_CUDA(cudaMemcpyAsync(h->scene_center, sc, sizeof(sc), cudaMemcpyHostToDevice, st));
    h->views.resize(V);
    int tile_off = 0;
    int64_t pix_off = 0;
    for (int v = 0; v < V; ++v) {
        svr_view_t w = views_in[v];
        w.tiles_x = (w.width + SVR_TILE - 1) / SVR_TILE;
        w.tiles_y = (w.height + SVR_TILE - 1) / SVR_TILE;
        w.tile_offset = tile_off;
        w.pix_offset = pix_off;
        w.w2c = h->mats + (size_t)v * 36;
        w.c2w = h->mats + (size_t)v * 36 + 16;
        w.bg = h->mats + (size_t)v * 36 + 32;
        tile_off += w.tiles_x * w.tiles_y;
        pix_off += (int64_t)w.width * w.height;
        h->views[v] = w;
    }
    h->tiles = tile_off;
    h->P = pix_off;

    // binning: pair order of the octree, record buffers sized for the views' record count
    size_t ws_bytes = 0;
    STEP_TRY(svr_rank_table_workspace_bytes(N, &ws_bytes));
    void* ws = nullptr;
    STEP_TRY(h->alloc(reinterpret_cast<uint8_t**>(&ws), (int64_t)ws_bytes));
    STEP_TRY(h->alloc(&h->pair_pos, 8ll * N));
    STEP_TRY(svr_pair_order_build(N, d.octpath, h->pair_pos, &h->key_bits, ws, ws_bytes, s));
    const int64_t M = (int64_t)N * V;
    STEP_TRY(h->alloc(&h->n_dup, M));
    STEP_TRY(h->alloc(reinterpret_cast<uint8_t**>(&h->geom), (int64_t)svr_geom_buffer_bytes(M)));
    h->capacity = d.record_capacity;
    if (h->capacity == 0) {
        STEP_TRY(svr_preprocess(h->views.data(), V, N, d.centers, d.lengths, d.is_leaf, d.octpath, h->n_dup, h->geom,
                                s));
        int64_t R = 0;
        uint64_t por = 0;
        STEP_TRY(svr_rendered_total(h->geom, &R, &por, s));
        h->capacity = std::max<int64_t>(R, 1);
    }
    h->bin_bytes = svr_binning_buffer_bytes(h->capacity, h->tiles);
    STEP_TRY(h->alloc(reinterpret_cast<uint8_t**>(&h->binning), (int64_t)h->bin_bytes));
    STEP_TRY(h->alloc(reinterpret_cast<uint8_t**>(&h->image), (int64_t)svr_image_buffer_bytes(h->P, h->tiles)));
    STEP_TRY(h->alloc(&h->all_idx, N));
    iota64_kernel<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(N, h->all_idx);
    svr_note_launch(1);
    STEP_CUDA(cudaGetLastError());

    // dense grid of the smoothness losses (src/utils/octree_utils.py:293-314, train.py:177-181)
    h->res = 1 << d.grid_res_pow2;
    h->vox_size_min_inv = (float)((double)h->res / (double)d.inside_extent);
    int64_t G = 0;
    size_t tws = std::max(svr_valid_table_workspace_bytes(N, 0), (size_t)16);
    void* tw = nullptr;
    STEP_CUDA(cudaMalloc(&tw, tws));
    int rc = svr_valid_table_count(N, d.centers, d.lengths, h->scene_center, d.inside_extent, d.grid_res_pow2,
                                   d.is_leaf, tw, &G, s);
    if (rc == SVR_OK && svr_valid_table_workspace_bytes(N, G) > tws) {
        void* tw2 = nullptr;
        const size_t need = svr_valid_table_workspace_bytes(N, G);
        cudaError_t e = cudaMalloc(&tw2, need);
        if (e == cudaSuccess) e = cudaMemcpyAsync(tw2, tw, tws, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaFree(tw);
        tw = tw2;
        if (e != cudaSuccess) { cudaFree(tw); return svr_fail(SVR_ERR_CUDA, "step: dense-grid table workspace"); }
    }
    if (rc != SVR_OK) { cudaFree(tw); return rc; }
    if (G >= (1ll << 31)) { cudaFree(tw); return svr_fail(SVR_ERR_CAPACITY, "step: dense-grid table too large"); }
    h->G = (int)G;
    const int64_t cells = (int64_t)h->res * h->res * h->res;
    rc = h->alloc(&h->grid_mask, cells);
    if (rc == SVR_OK) rc = h->alloc(&h->grid_keys, G);
    if (rc == SVR_OK) rc = h->alloc(&h->grid2voxel, G);
    if (rc == SVR_OK) rc = svr_valid_table_fill(N, d.centers, d.lengths, h->scene_center, d.inside_extent,
                                                d.grid_res_pow2, d.is_leaf, G, tw, h->grid_mask, h->grid_keys,
                                                h->grid2voxel, s);
    if (rc == SVR_OK) { cudaError_t e = cudaStreamSynchronize(st); if (e != cudaSuccess) rc = svr_fail(SVR_ERR_CUDA, "step: table fill"); }
    cudaFree(tw);
    STEP_TRY(rc);
    STEP_TRY(h->alloc(&h->status, 1));
    STEP_CUDA(cudaMemsetAsync(h->status, 0, sizeof(uint32_t), st));
    STEP_TRY(h->alloc(&h->grid_index, cells));
    if (h->G > 0) STEP_TRY(svr_grid_index_build(h->G, h->grid_keys, h->res, h->grid_index, h->status, s));
    STEP_TRY(h->alloc(&h->vcoord, 3ll * N));
    STEP_TRY(h->alloc(&h->vsize, N));
    grid_coords_kernel<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(
        N, d.centers, d.lengths, make_float3(d.scene_center[0], d.scene_center[1], d.scene_center[2]),
        d.inside_extent, (float)h->res, h->vcoord, h->vsize);
    svr_note_launch(1);
    STEP_CUDA(cudaGetLastError());

    // per-step state and planes
    STEP_TRY(h->alloc(&h->geos, 8ll * N));
    STEP_TRY(h->alloc(&h->rgbs, 3ll * V * N));
    STEP_TRY(h->alloc(&h->drgbs, 3ll * V * N));
    STEP_TRY(h->alloc(&h->dvox, 12ll * N));
    STEP_TRY(h->alloc(&h->ds, 1));
    for (int p = 0; p < kPlanes; ++p) {
        if (p == kPlaneGT && !(d.lambda_R_concen > 0.f)) continue;
        STEP_TRY(h->alloc(&h->plane[p], kPlaneWidth[p] * h->P));
        STEP_CUDA(cudaMemsetAsync(h->plane[p], 0, (size_t)kPlaneWidth[p] * h->P * sizeof(float), st));
    }

    // gradients: one flat buffer, every parameter's view on a 64-float (256-byte) boundary
    h->numel[0] = d.n_grid;
    h->numel[1] = 3ll * N;
    h->numel[2] = 3ll * N * (h->M_sh - 1);
    int64_t off[3], total = 0;
    for (int k = 0; k < 3; ++k) { off[k] = total; total += round_up(h->numel[k], 64); }
    h->n_flat = std::max<int64_t>(total, 1);
    STEP_TRY(h->alloc(&h->grad_flat, h->n_flat));
    STEP_CUDA(cudaMemsetAsync(h->grad_flat, 0, (size_t)h->n_flat * sizeof(float), st));
    for (int k = 0; k < 3; ++k) h->grad[k] = h->grad_flat + off[k];

    // Adam: f32 moments, per-step coefficient table, device step counter
    h->rows = d.adam_rows > 0 ? d.adam_rows : (1 << 20);
    std::vector<float> tab((size_t)h->rows * 2);
    for (int k = 0; k < 3; ++k) {
        STEP_TRY(h->alloc(&h->adam_m[k], h->numel[k]));
        STEP_TRY(h->alloc(&h->adam_v[k], h->numel[k]));
        STEP_CUDA(cudaMemsetAsync(h->adam_m[k], 0, (size_t)std::max<int64_t>(h->numel[k], 1) * sizeof(float), st));
        STEP_CUDA(cudaMemsetAsync(h->adam_v[k], 0, (size_t)std::max<int64_t>(h->numel[k], 1) * sizeof(float), st));
        STEP_TRY(h->alloc(&h->coef[k], 2 * h->rows));
        STEP_TRY(svr_adam_coef_table(0, d.lr[k], d.beta1, d.beta2, h->rows, tab.data()));
        STEP_CUDA(cudaMemcpyAsync(h->coef[k], tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice, st));
        STEP_CUDA(cudaStreamSynchronize(st));   // `tab` is reused by the next parameter
    }
    STEP_TRY(h->alloc(&h->step_dev, 1));
    STEP_CUDA(cudaMemsetAsync(h->step_dev, 0, sizeof(int64_t), st));
    STEP_CUDA(cudaStreamCreateWithFlags(&h->cap, cudaStreamNonBlocking));
    STEP_CUDA(cudaStreamSynchronize(st));
    return SVR_OK;
}

static void drop_graphs(svr_step* h)
{
    for (auto& e : h->exec)
        if (e) { cudaGraphExecDestroy(e); e = nullptr; }
}

extern "C" int svr_step_destroy(svr_step_t* h)
{
    if (!h) return SVR_OK;
    // the caller's streams may still run this step's graphs or launches: wait for the device
    cudaDeviceSynchronize();
    drop_graphs(h);
    for (void* p : h->allocs) cudaFree(p);
    if (h->cap) cudaStreamDestroy(h->cap);
    delete h;
    return SVR_OK;
}

extern "C" int svr_step_create(const svr_step_desc_t* desc, const svr_view_t* views_host, int n_views, void* stream,
                               svr_step_t** out_host)
{
    if (!out_host) return svr_fail(SVR_ERR_ARG, "step: null output handle");
    *out_host = nullptr;
    STEP_TRY(check_desc(desc, views_host, n_views));
    svr_step* h = new svr_step();
    h->d = *desc;
    h->V = n_views;
    h->N = desc->n_vox;
    const int rc = build(h, views_host, (cudaStream_t)stream);
    if (rc != SVR_OK) {
        const std::string msg = svr_last_error();
        cudaStreamSynchronize((cudaStream_t)stream);
        svr_step_destroy(h);
        return svr_fail(rc, msg.c_str());
    }
    *out_host = h;
    return SVR_OK;
}

// ------------------------------------------------------------------ run / capture / query
extern "C" int svr_step_run(svr_step_t* h, int phases, void* stream)
{
    if (!h) return svr_fail(SVR_ERR_ARG, "step: null handle");
    if (phases < 1 || phases > 3) return svr_fail(SVR_ERR_ARG, "step: phases must be 1, 2 or 3");
    cudaStream_t st = (cudaStream_t)stream;
    for (int p = 0; p < 2; ++p) {
        if (!(phases & (1 << p))) continue;
        if (h->exec[p]) STEP_CUDA(cudaGraphLaunch(h->exec[p], st));
        else STEP_TRY(run_phase(h, p, st));
    }
    return SVR_OK;
}

extern "C" int svr_step_capture(svr_step_t* h, void* stream)
{
    if (!h) return svr_fail(SVR_ERR_ARG, "step: null handle");
    cudaStream_t st = (cudaStream_t)stream;
    drop_graphs(h);
    // one eager pass of the gradient phase sets the kernels' attributes outside the capture
    // and counts the launches; it changes no parameter (Adam is not run)
    STEP_TRY(run_phase(h, 0, st));
    STEP_CUDA(cudaStreamSynchronize(st));
    for (int p = 0; p < 2; ++p) {
        const long long n0 = svr_kernel_launches();
        STEP_CUDA(cudaStreamBeginCapture(h->cap, cudaStreamCaptureModeThreadLocal));
        const int rc = p == 0 ? phase_grads(h, h->cap) : phase_adam(h, h->cap);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(h->cap, &g);
        if (rc != SVR_OK || e != cudaSuccess) {
            const std::string msg = rc != SVR_OK ? std::string(svr_last_error()) : cudaGetErrorString(e);
            if (g) cudaGraphDestroy(g);
            drop_graphs(h);
            return svr_fail(rc != SVR_OK ? rc : SVR_ERR_CUDA, ("step capture: " + msg).c_str());
        }
        h->kernels[p] = svr_kernel_launches() - n0;
        const cudaError_t ei = cudaGraphInstantiate(&h->exec[p], g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            drop_graphs(h);
            return svr_fail(SVR_ERR_CUDA, (std::string("step capture: ") + cudaGetErrorString(ei)).c_str());
        }
    }
    // the graphs are uploaded before their first launch on the caller's stream
    for (int p = 0; p < 2; ++p) STEP_CUDA(cudaGraphUpload(h->exec[p], st));
    STEP_CUDA(cudaStreamSynchronize(st));
    return SVR_OK;
}

extern "C" int svr_step_buffer(const svr_step_t* h, int which, void** ptr_host, int64_t* count_host)
{
    if (!h || !ptr_host || !count_host) return svr_fail(SVR_ERR_ARG, "step: null argument");
    void* p = nullptr;
    int64_t n = 0;
    switch (which) {
    case SVR_STEP_COLOR: case SVR_STEP_DEPTH: case SVR_STEP_NORMAL: case SVR_STEP_T:
    case SVR_STEP_DCOLOR: case SVR_STEP_DDEPTH: case SVR_STEP_DNORMAL: case SVR_STEP_DT: case SVR_STEP_GT:
        p = h->plane[which];
        n = p ? kPlaneWidth[which] * h->P : 0;
        break;
    case SVR_STEP_GRAD_FLAT: p = h->grad_flat; n = h->n_flat; break;
    case SVR_STEP_GRAD_GRID: p = h->grad[0]; n = h->numel[0]; break;
    case SVR_STEP_GRAD_SH0: p = h->grad[1]; n = h->numel[1]; break;
    case SVR_STEP_GRAD_SHS: p = h->grad[2]; n = h->numel[2]; break;
    case SVR_STEP_DVOX: p = h->dvox; n = 12ll * h->N; break;
    case SVR_STEP_DS: p = h->ds; n = 1; break;
    case SVR_STEP_STEP: p = h->step_dev; n = 1; break;
    default: return svr_fail(SVR_ERR_ARG, "step: unknown buffer");
    }
    *ptr_host = p;
    *count_host = n;
    return SVR_OK;
}

extern "C" int svr_step_info(const svr_step_t* h, int64_t* info)
{
    if (!h || !info) return svr_fail(SVR_ERR_ARG, "step: null argument");
    info[0] = h->P;
    info[1] = h->capacity;
    info[2] = h->tiles;
    info[3] = h->G;
    info[4] = h->n_flat;
    info[5] = h->V;
    info[6] = h->kernels[0] + h->kernels[1];
    info[7] = (h->exec[0] && h->exec[1]) ? 1 : 0;
    return SVR_OK;
}

extern "C" int svr_step_status(const svr_step_t* h, uint32_t* raster_host, uint32_t* other_host, void* stream)
{
    if (!h || !raster_host || !other_host) return svr_fail(SVR_ERR_ARG, "step: null argument");
    cudaStream_t st = (cudaStream_t)stream;
    STEP_TRY(svr_read_status(h->image, h->P, h->tiles, raster_host, stream));
    STEP_CUDA(cudaMemcpyAsync(other_host, h->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    STEP_CUDA(cudaStreamSynchronize(st));
    return SVR_OK;
}
