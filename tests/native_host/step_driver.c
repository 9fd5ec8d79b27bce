/*
 * A host program in plain C that drives the batched training step through the C ABI only
 * (include/svraster_b200.h, libsvraster_b200.so and the CUDA runtime; no Python in the process).
 *
 *   step_driver --layout
 *       prints sizeof(svr_step_desc_t) and the offset of every field (no CUDA call), so that
 *       other bindings can check their mirror of the struct.
 *   step_driver <input> <output> <steps> <eager|graph>
 *       reads a scene, its views and one set of upstream gradient planes from <input>, creates
 *       the step, runs <steps> steps (copying the upstream planes from host memory before each
 *       one) and writes the step's outputs and the updated parameters to <output>.
 *
 * Input (little-endian, packed): double header[16] = {N, n_grid, sh_degree, V, grid_res_pow2,
 * seed, inside_extent, s_val, lambda_ls, lambda_ge, lr_grid, lr_sh0, lr_shs, beta1, beta2, eps},
 * then octpath i64[N], centers f32[N*3], lengths f32[N], is_leaf u8[N], vox_key i64[N*8],
 * grid f32[n_grid], sh0 f32[N*3], shs f32[N*(M-1)*3] (M = (sh_degree+1)^2), per view
 * {i32 width, height; f32 tanfovx, tanfovy, cx, cy, near; f32 w2c[16], c2w[16]}, then
 * dcolor f32[3P], ddepth f32[4P], dnormal f32[3P] (P = total pixels).
 * Output: i64 info[8], u32 status[2], then color f32[3P], T f32[P], grad_flat f32[info[4]],
 * grid f32[n_grid], sh0 f32[N*3], shs f32[N*(M-1)*3].
 */
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "svraster_b200.h"

static int fail(const char* what, int rc)
{
    fprintf(stderr, "step_driver: %s failed (%d): %s\n", what, rc, svr_last_error());
    return 1;
}

#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { \
    fprintf(stderr, "step_driver: %s: %s\n", #x, cudaGetErrorString(e_)); return 1; } } while (0)
#define SV(x, what) do { int r_ = (x); if (r_ != SVR_OK) return fail(what, r_); } while (0)

static void* read_block(FILE* f, size_t bytes)
{
    void* p = malloc(bytes ? bytes : 1);
    if (p && bytes && fread(p, 1, bytes, f) != bytes) { free(p); return NULL; }
    return p;
}

static int to_device(void** dst, const void* src, size_t bytes)
{
    CK(cudaMalloc(dst, bytes ? bytes : 16));
    if (bytes) CK(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
    return 0;
}

static int print_layout(void)
{
#define OFF(f) printf("%s %zu\n", #f, offsetof(svr_step_desc_t, f))
    printf("sizeof %zu\n", sizeof(svr_step_desc_t));
    OFF(n_vox); OFF(sh_degree); OFF(sh_bf16); OFF(grid_res_pow2); OFF(octpath); OFF(centers); OFF(lengths);
    OFF(is_leaf); OFF(vox_key); OFF(grid); OFF(sh0); OFF(shs); OFF(n_grid); OFF(s_val); OFF(scene_center);
    OFF(inside_extent); OFF(lambda_ls); OFF(lambda_ge); OFF(lambda_R_concen); OFF(lr); OFF(beta1); OFF(beta2);
    OFF(eps); OFF(seed); OFF(adam_rows); OFF(record_capacity);
#undef OFF
    printf("view_sizeof %zu\n", sizeof(svr_view_t));
    return 0;
}

int main(int argc, char** argv)
{
    if (argc == 2 && strcmp(argv[1], "--layout") == 0) return print_layout();
    if (argc != 5) {
        fprintf(stderr, "usage: step_driver --layout | <input> <output> <steps> <eager|graph>\n");
        return 2;
    }
    const int steps = atoi(argv[3]);
    const int graph = strcmp(argv[4], "graph") == 0;
    FILE* f = fopen(argv[1], "rb");
    if (!f) { perror(argv[1]); return 1; }
    double hd[16];
    if (fread(hd, sizeof(double), 16, f) != 16) { fprintf(stderr, "short header\n"); return 1; }
    const int64_t N = (int64_t)hd[0], n_grid = (int64_t)hd[1];
    const int deg = (int)hd[2], V = (int)hd[3];
    const int M = (deg + 1) * (deg + 1);
    if (N <= 0 || V <= 0 || V > SVR_MAX_VIEWS) { fprintf(stderr, "bad header\n"); return 1; }

    const size_t sz_path = 8 * N, sz_c = 12 * N, sz_l = 4 * N, sz_leaf = N, sz_key = 64 * N;
    const size_t sz_grid = 4 * n_grid, sz_sh0 = 12 * N, sz_shs = 12 * N * (M - 1);
    void* h_path = read_block(f, sz_path); void* h_c = read_block(f, sz_c); void* h_l = read_block(f, sz_l);
    void* h_leaf = read_block(f, sz_leaf); void* h_key = read_block(f, sz_key); void* h_grid = read_block(f, sz_grid);
    void* h_sh0 = read_block(f, sz_sh0); void* h_shs = read_block(f, sz_shs);
    if (!h_path || !h_c || !h_l || !h_leaf || !h_key || !h_grid || !h_sh0 || !h_shs) {
        fprintf(stderr, "short scene\n"); return 1;
    }
    svr_view_t views[SVR_MAX_VIEWS];
    memset(views, 0, sizeof(views));
    int64_t P = 0;
    for (int v = 0; v < V; ++v) {
        int32_t wh[2];
        float cam[5], mats[32];
        if (fread(wh, 4, 2, f) != 2 || fread(cam, 4, 5, f) != 5 || fread(mats, 4, 32, f) != 32) {
            fprintf(stderr, "short view\n"); return 1;
        }
        views[v].width = wh[0]; views[v].height = wh[1];
        views[v].tanfovx = cam[0]; views[v].tanfovy = cam[1]; views[v].cx = cam[2]; views[v].cy = cam[3];
        views[v].near_plane = cam[4];
        void* d_w2c = NULL; void* d_c2w = NULL;
        if (to_device(&d_w2c, mats, 64) || to_device(&d_c2w, mats + 16, 64)) return 1;
        views[v].w2c = (const float*)d_w2c; views[v].c2w = (const float*)d_c2w; views[v].bg = NULL;
        P += (int64_t)wh[0] * wh[1];
    }
    float* up[3];
    const int upw[3] = {3, 4, 3};
    for (int k = 0; k < 3; ++k) {
        up[k] = (float*)read_block(f, (size_t)upw[k] * P * 4);
        if (!up[k]) { fprintf(stderr, "short upstream planes\n"); return 1; }
    }
    fclose(f);

    void *d_path, *d_c, *d_l, *d_leaf, *d_key, *d_grid, *d_sh0, *d_shs, *d_s;
    const float s_val = (float)hd[7];
    if (to_device(&d_path, h_path, sz_path) || to_device(&d_c, h_c, sz_c) || to_device(&d_l, h_l, sz_l) ||
        to_device(&d_leaf, h_leaf, sz_leaf) || to_device(&d_key, h_key, sz_key) ||
        to_device(&d_grid, h_grid, sz_grid) || to_device(&d_sh0, h_sh0, sz_sh0) ||
        to_device(&d_shs, h_shs, sz_shs) || to_device(&d_s, &s_val, 4))
        return 1;

    svr_step_desc_t d;
    memset(&d, 0, sizeof(d));
    d.n_vox = (int32_t)N; d.sh_degree = deg; d.sh_bf16 = 0; d.grid_res_pow2 = (int32_t)hd[4];
    d.octpath = (const int64_t*)d_path; d.centers = (const float*)d_c; d.lengths = (const float*)d_l;
    d.is_leaf = (const uint8_t*)d_leaf; d.vox_key = (const int64_t*)d_key;
    d.grid = (float*)d_grid; d.sh0 = d_sh0; d.shs = d_shs; d.n_grid = n_grid; d.s_val = (const float*)d_s;
    d.inside_extent = (float)hd[6];
    d.lambda_ls = (float)hd[8]; d.lambda_ge = (float)hd[9];
    d.lr[0] = hd[10]; d.lr[1] = hd[11]; d.lr[2] = hd[12];
    d.beta1 = hd[13]; d.beta2 = hd[14]; d.eps = (float)hd[15];
    d.seed = (int32_t)hd[5];

    cudaStream_t st;
    CK(cudaStreamCreate(&st));
    svr_step_t* step = NULL;
    SV(svr_step_create(&d, views, V, st, &step), "svr_step_create");
    float* planes[3];
    int64_t n = 0;
    const int up_buf[3] = {SVR_STEP_DCOLOR, SVR_STEP_DDEPTH, SVR_STEP_DNORMAL};
    for (int k = 0; k < 3; ++k) SV(svr_step_buffer(step, up_buf[k], (void**)&planes[k], &n), "svr_step_buffer");
    if (graph) SV(svr_step_capture(step, st), "svr_step_capture");
    for (int it = 0; it < steps; ++it) {
        for (int k = 0; k < 3; ++k)
            CK(cudaMemcpyAsync(planes[k], up[k], (size_t)upw[k] * P * 4, cudaMemcpyHostToDevice, st));
        SV(svr_step_run(step, SVR_STEP_GRADS | SVR_STEP_ADAM, st), "svr_step_run");
    }
    CK(cudaStreamSynchronize(st));

    int64_t info[8];
    uint32_t status[2];
    SV(svr_step_info(step, info), "svr_step_info");
    SV(svr_step_status(step, &status[0], &status[1], st), "svr_step_status");
    FILE* o = fopen(argv[2], "wb");
    if (!o) { perror(argv[2]); return 1; }
    fwrite(info, 8, 8, o);
    fwrite(status, 4, 2, o);
    const int outs[3] = {SVR_STEP_COLOR, SVR_STEP_T, SVR_STEP_GRAD_FLAT};
    for (int k = 0; k < 3; ++k) {
        void* p = NULL;
        SV(svr_step_buffer(step, outs[k], &p, &n), "svr_step_buffer");
        float* h = (float*)malloc((size_t)n * 4);
        CK(cudaMemcpy(h, p, (size_t)n * 4, cudaMemcpyDeviceToHost));
        fwrite(h, 4, (size_t)n, o);
        free(h);
    }
    const void* params[3] = {d_grid, d_sh0, d_shs};
    const size_t psz[3] = {sz_grid, sz_sh0, sz_shs};
    for (int k = 0; k < 3; ++k) {
        void* h = malloc(psz[k] ? psz[k] : 1);
        if (psz[k]) CK(cudaMemcpy(h, params[k], psz[k], cudaMemcpyDeviceToHost));
        fwrite(h, 1, psz[k], o);
        free(h);
    }
    fclose(o);
    SV(svr_step_destroy(step), "svr_step_destroy");
    CK(cudaStreamDestroy(st));
    printf("steps %d mode %s kernels_per_step %lld records %lld status %u %u\n", steps, argv[4],
           (long long)info[6], (long long)info[1], status[0], status[1]);
    return 0;
}
