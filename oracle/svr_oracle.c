/*
 * CPU oracle for the sparse-voxel SDF rasterizer path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference algorithms (alvin0808/svraster, SDF mode),
 * single precision, same expression order as the reference so that compilers that
 * contract a*b+c the same way produce the same bits.  Only the tests, the smoke check
 * and the CPU-baseline leg of the benchmark may call it; the product never does.
 *
 * Every function cites the reference file:line it restates.  Parity of this file with
 * the reference itself is pinned by golden vectors produced by the reference's own CUDA
 * extension (tests/golden/).
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* The render math is typed on `real`: float reproduces the reference's single-precision
 * arithmetic (the parity checker); -DSVO_REAL_DOUBLE builds the FP64 per-ray oracle used
 * for finite-difference gradient checks.  Preprocess and binning are always float (their
 * integer outputs must match the reference bit for bit). */
#ifdef SVO_REAL_DOUBLE
typedef double real;
#define EXPR exp
#define SQRTR sqrt
#define FABSR fabs
#else
typedef float real;
#define EXPR expf
#define SQRTR sqrtf
#define FABSR fabsf
#endif

#define TILE 16
#define NUM_BIT_ORDER_RANK 48
#define MAX_LEVELS 16
#define MIN_ALPHA 0.00001f
#define EARLY_STOP_T 0.0001f

/* Host threads used by the render loops (tiles are independent; the adjoint scatters with
 * atomics).  Default 1 so results are deterministic; the CPU baseline raises it. */
static int g_threads = 1;
void svo_set_threads(int n) { g_threads = n > 0 ? n : 1; }

/* Optional pixel mask (uint8[H*W], nonzero = render) for the per-ray checks: masked-out
 * pixels are skipped by both render passes (their outputs stay as the caller initialised
 * them; they contribute no gradient).  NULL renders every pixel. */
static const uint8_t* g_pixel_mask = NULL;
void svo_set_pixel_mask(const uint8_t* mask) { g_pixel_mask = mask; }

/* Optional decision trace for the parity tests (uint8[H*W] per pixel, uint8[N] per voxel).
 * The forward ORs into the pixel trace: TR_ALPHA an evaluated pair whose alpha lies within
 * TR_ALPHA_BAND of MIN_ALPHA (kept in one precision, dropped in another); TR_STOP an accepted
 * pair that left T within TR_STOP_BAND of the early-stop threshold; TR_MEDIAN a median-depth
 * decision with T within TR_MED_BAND of 0.5.  The adjoint ORs TR_ADJ for a pair whose
 * recomputed alpha lies within TR_ALPHA_BAND of MIN_ALPHA or whose depth sub-segment raw
 * alpha lies within TR_RAW_BAND of 0 (the derivative switch), and marks in the voxel trace
 * every voxel that a pixel with a forward flag contributes gradient to.  The bands are a few float32
 * ulps of the quantity compared, scaled up by the cancellation in alpha. */
#define TR_ALPHA 1
#define TR_STOP 2
#define TR_MEDIAN 4
#define TR_ADJ 8
#define TR_ALPHA_BAND 5e-7
#define TR_STOP_BAND 1e-7
#define TR_MED_BAND 5e-6
#define TR_RAW_BAND 1e-6
static uint8_t* g_trace = NULL;
static uint8_t* g_vox_trace = NULL;
void svo_set_trace(uint8_t* pixel_trace, uint8_t* voxel_trace) { g_trace = pixel_trace; g_vox_trace = voxel_trace; }
/* Optional: the adjoint also adds |term| of every pair's 12 gradient terms into abs_sum[N,12]
 * (the scale against which a sum of those terms computed in another order or precision is
 * compared).  Same type as the build's render math; NULL switches it off. */
static void* g_abs_sum = NULL;
void svo_set_abs_sum(void* abs_sum) { g_abs_sum = abs_sum; }
static inline double dabs(double x) { return x < 0 ? -x : x; }
int svo_get_threads(void) { return g_threads; }

typedef struct { float x, y, z; } f3;

static inline f3 mk(float x, float y, float z) { f3 r = {x, y, z}; return r; }
static inline f3 add(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline f3 sub(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline f3 adds(f3 a, float b) { return mk(a.x + b, a.y + b, a.z + b); }
static inline f3 subs(f3 a, float b) { return mk(a.x - b, a.y - b, a.z - b); }
static inline f3 mul(f3 a, f3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline f3 muls(f3 a, float b) { return mk(a.x * b, a.y * b, a.z * b); }
static inline float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float minf(float a, float b) { return a < b ? a : b; }
static inline float maxf(float a, float b) { return a > b ? a : b; }

typedef struct { real x, y, z; } r3;
static inline r3 rk(real x, real y, real z) { r3 r = {x, y, z}; return r; }
static inline r3 radd(r3 a, r3 b) { return rk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline r3 rsub(r3 a, r3 b) { return rk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline r3 radds(r3 a, real b) { return rk(a.x + b, a.y + b, a.z + b); }
static inline r3 rsubs(r3 a, real b) { return rk(a.x - b, a.y - b, a.z - b); }
static inline r3 rmul(r3 a, r3 b) { return rk(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline r3 rmuls(r3 a, real b) { return rk(a.x * b, a.y * b, a.z * b); }
static inline real rdot(r3 a, r3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline real rmin(real a, real b) { return a < b ? a : b; }
static inline real rmax(real a, real b) { return a > b ? a : b; }

/* cuda/src/auxiliary.h:212-243 -- 3x4 row-major use of a 4x4 matrix */
static inline f3 transform_3x4(const float* m, f3 p) {
    return mk(m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3],
              m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
              m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]);
}
static inline f3 rotate_3x4(const float* m, f3 p) {
    return mk(m[0] * p.x + m[1] * p.y + m[2] * p.z,
              m[4] * p.x + m[5] * p.y + m[6] * p.z,
              m[8] * p.x + m[9] * p.y + m[10] * p.z);
}

/* cuda/src/auxiliary.h:251-264 */
static inline void ray_aabb(f3 c, float l, f3 ro, f3 rd_inv, float* a, float* b) {
    float r = 0.5f * l;
    f3 dir = sub(c, ro);
    f3 c0_ = mul(subs(dir, r), rd_inv);
    f3 c1_ = mul(adds(dir, r), rd_inv);
    f3 c0 = mk(minf(c0_.x, c1_.x), minf(c0_.y, c1_.y), minf(c0_.z, c1_.z));
    f3 c1 = mk(maxf(c0_.x, c1_.x), maxf(c0_.y, c1_.y), maxf(c0_.z, c1_.z));
    *a = maxf(maxf(c0.x, c0.y), c0.z);
    *b = minf(minf(c1.x, c1.y), c1.z);
}

/* cuda/src/auxiliary.h:319-333 (corner index x<<2 | y<<1 | z) */
static inline void tri_w(f3 q, float w[8]) {
    float wx0 = 1.f - q.x, wx1 = q.x, wy0 = 1.f - q.y, wy1 = q.y, wz0 = 1.f - q.z, wz1 = q.z;
    w[0] = wx0 * wy0 * wz0; w[1] = wx0 * wy0 * wz1; w[2] = wx0 * wy1 * wz0; w[3] = wx0 * wy1 * wz1;
    w[4] = wx1 * wy0 * wz0; w[5] = wx1 * wy0 * wz1; w[6] = wx1 * wy1 * wz0; w[7] = wx1 * wy1 * wz1;
}
static inline float interp8(const float* g, const float* w) {
    float s = 0.f;
    for (int i = 0; i < 8; ++i) s += g[i] * w[i];
    return s;
}
static inline float sigm(float s, float x) { return 1.f / (1.f + expf(-s * x)); }
static inline float rnorm3(float x, float y, float z) { return 1.f / sqrtf(x * x + y * y + z * z + 1e-15f); }

/* ------------------------------------------------------------------ preprocess
 * cuda/src/preprocess.cu:36-154 (perspective camera); host derivations :196-198. */
/* The projection is spelled out operation by operation, with contraction off for this
 * function and the bbox step fused explicitly, the same rounding the library's preprocess
 * spells out: integer bboxes sit on pixel rounding boundaries, so both sides fix it rather
 * than leave it to a compiler. */
__attribute__((optimize("fp-contract=off")))
void svo_preprocess(int P, int W, int H, float tanfovx, float tanfovy, float cx, float cy,
                    const float* w2c, const float* c2w, float near,
                    const float* centers, const float* lengths, const uint8_t* is_leaf,
                    int32_t* out_ndup, uint32_t* bboxes, uint32_t* bits)
{
    const int gx = (W + TILE - 1) / TILE, gy = (H + TILE - 1) / TILE;
    const float focal_x = 0.5f * W / tanfovx;
    const float focal_y = 0.5f * H / tanfovy;
    const float rox = c2w[3], roy = c2w[7], roz = c2w[11];
    const float* m = w2c;
    for (int i = 0; i < P; ++i) {
        out_ndup[i] = 0; bboxes[2 * i] = 0; bboxes[2 * i + 1] = 0; bits[i] = 0;
        if (is_leaf[i] == 0) continue;
        const float cxv = centers[3 * i], cyv = centers[3 * i + 1], czv = centers[3 * i + 2];
        const float r = 0.5f * lengths[i];
        const float dxr = cxv - rox, dyr = cyv - roy, dzr = czv - roz;
        const float d2 = (dxr * dxr + dyr * dyr) + dzr * dzr;
        if (d2 < near * near) continue;
        uint32_t qb = 0;
        float mnx = 1e9f, mny = 1e9f, mxx = -1e9f, mxy = -1e9f;
        for (int k = 0; k < 8; ++k) {
            const float sx = (float)(((k & 4) >> 2) * 2 - 1), sy = (float)(((k & 2) >> 1) * 2 - 1);
            const float sz = (float)((k & 1) * 2 - 1);
            const float wx = cxv + r * sx, wy = cyv + r * sy, wz = czv + r * sz;   /* exact: s = +-1 */
            const float X = ((m[0] * wx + m[1] * wy) + m[2] * wz) + m[3];
            const float Y = ((m[4] * wx + m[5] * wy) + m[6] * wz) + m[7];
            const float Z = ((m[8] * wx + m[9] * wy) + m[10] * wz) + m[11];
            if (Z < near) continue;
            const float iz = 1.0f / Z;
            const float u = X * iz, v = Y * iz;
            const int q = ((wx < rox) << 2) | ((wy < roy) << 1) | (wz < roz);
            mnx = minf(mnx, u); mny = minf(mny, v); mxx = maxf(mxx, u); mxy = maxf(mxy, v);
            qb |= 1u << q;
        }
        const float cxh = cx - 0.5f, cyh = cy - 0.5f;
        const float bminx = maxf(fmaf(focal_x, mnx, cxh), 0.0f), bminy = maxf(fmaf(focal_y, mny, cyh), 0.0f);
        const float bmaxx = minf(fmaf(focal_x, mxx, cxh), (float)W), bmaxy = minf(fmaf(focal_y, mxy, cyh), (float)H);
        if (bminx > bmaxx || bminy > bmaxy) continue;
        uint32_t b0 = (((uint32_t)lrintf(bminx)) << 16) | ((uint32_t)lrintf(bminy));
        uint32_t b1 = (((uint32_t)lrintf(bmaxx)) << 16) | ((uint32_t)lrintf(bmaxy));
        /* auxiliary.h:138-152 */
        int x0 = (int)(b0 >> 16), y0 = (int)(b0 & 0xFFFF), x1 = (int)(b1 >> 16), y1 = (int)(b1 & 0xFFFF);
        int tx0 = x0 / TILE, ty0 = y0 / TILE, tx1 = x1 / TILE, ty1 = y1 / TILE;
        tx0 = tx0 > gx - 1 ? gx - 1 : tx0; tx1 = tx1 > gx - 1 ? gx - 1 : tx1;
        ty0 = ty0 > gy - 1 ? gy - 1 : ty0; ty1 = ty1 > gy - 1 ? gy - 1 : ty1;
        int tiles = (1 + ty1 - ty0) * (1 + tx1 - tx0);
        out_ndup[i] = tiles * __builtin_popcount(qb);
        bboxes[2 * i] = b0; bboxes[2 * i + 1] = b1; bits[i] = qb;
    }
}

/* ------------------------------------------------------------------ binning
 * cuda/src/forward.cu:749-829 (duplicateWithKeys, identifyTileRanges) and the stable
 * CUB radix sort of forward.cu:920-925.  Keys are [tile | octpath ^ repeat3(q)],
 * values are [q << 29 | voxel id]. */
typedef struct { uint64_t key; uint32_t val; uint32_t pos; } rec_t;

static int cmp_rec(const void* a, const void* b) {
    const rec_t* x = (const rec_t*)a; const rec_t* y = (const rec_t*)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->pos < y->pos ? -1 : (x->pos > y->pos);
}

static uint64_t repeat3(uint64_t q) {
    uint64_t v = 0;
    for (int l = 0; l < MAX_LEVELS; ++l) v = (v << 3) | q;
    return v;
}

int64_t svo_num_rendered(int P, const int32_t* ndup) {
    int64_t s = 0;
    for (int i = 0; i < P; ++i) s += ndup[i];
    return s;
}

void svo_binning(int P, int W, int H, const int64_t* octpath, const int32_t* ndup,
                 const uint32_t* bboxes, const uint32_t* bits,
                 uint64_t* keys_out, uint32_t* vals_out, uint32_t* ranges /* 2 per tile */)
{
    const int gx = (W + TILE - 1) / TILE, gy = (H + TILE - 1) / TILE;
    int64_t R = svo_num_rendered(P, ndup);
    rec_t* rec = (rec_t*)malloc(sizeof(rec_t) * (R > 0 ? R : 1));
    int64_t off = 0;
    for (int i = 0; i < P; ++i) {
        if (ndup[i] == 0) continue;
        uint32_t b0 = bboxes[2 * i], b1 = bboxes[2 * i + 1];
        int x0 = (int)(b0 >> 16) / TILE, y0 = (int)(b0 & 0xFFFF) / TILE;
        int x1 = (int)(b1 >> 16) / TILE, y1 = (int)(b1 & 0xFFFF) / TILE;
        x0 = x0 > gx - 1 ? gx - 1 : x0; x1 = x1 > gx - 1 ? gx - 1 : x1;
        y0 = y0 > gy - 1 ? gy - 1 : y0; y1 = y1 > gy - 1 ? gy - 1 : y1;
        for (int q = 0; q < 8; ++q) {
            if (!(bits[i] & (1u << q))) continue;
            uint64_t rank = (uint64_t)octpath[i] ^ repeat3((uint64_t)q);
            for (int y = y0; y <= y1; ++y)
                for (int x = x0; x <= x1; ++x) {
                    uint64_t tile = (uint64_t)(y * gx + x);
                    rec[off].key = (tile << NUM_BIT_ORDER_RANK) | rank;
                    rec[off].val = ((uint32_t)q << 29) | (uint32_t)i;
                    rec[off].pos = (uint32_t)off;
                    off++;
                }
        }
    }
    qsort(rec, (size_t)R, sizeof(rec_t), cmp_rec);
    const int T = gx * gy;
    memset(ranges, 0, sizeof(uint32_t) * 2 * T);
    for (int64_t k = 0; k < R; ++k) {
        keys_out[k] = rec[k].key; vals_out[k] = rec[k].val;
        uint32_t t = (uint32_t)(rec[k].key >> NUM_BIT_ORDER_RANK);
        if (k == 0 || (uint32_t)(rec[k - 1].key >> NUM_BIT_ORDER_RANK) != t) ranges[2 * t] = (uint32_t)k;
        if (k == R - 1 || (uint32_t)(rec[k + 1].key >> NUM_BIT_ORDER_RANK) != t) ranges[2 * t + 1] = (uint32_t)(k + 1);
    }
    free(rec);
}

/* ------------------------------------------------------------------ render forward
 * cuda/src/forward.cu:41-564, SDF density (forward.cu:255-306), triinterp with n_samp
 * samples, mean depth (:345-379), linear normal (:420-434), median depth refinement
 * (:450-521).  Pixel (px,py) of tile (tx,ty); warp packing does not change results. */
static inline void rray_aabb(r3 c, real l, r3 ro, r3 rd_inv, real* a, real* b) {
    real r = (real)0.5f * l;
    r3 dir = rsub(c, ro);
    r3 c0_ = rmul(rsubs(dir, r), rd_inv);
    r3 c1_ = rmul(radds(dir, r), rd_inv);
    r3 c0 = rk(rmin(c0_.x, c1_.x), rmin(c0_.y, c1_.y), rmin(c0_.z, c1_.z));
    r3 c1 = rk(rmax(c0_.x, c1_.x), rmax(c0_.y, c1_.y), rmax(c0_.z, c1_.z));
    *a = rmax(rmax(c0.x, c0.y), c0.z);
    *b = rmin(rmin(c1.x, c1.y), c1.z);
}
static inline void rtri_w(r3 q, real w[8]) {
    real wx0 = 1.f - q.x, wx1 = q.x, wy0 = 1.f - q.y, wy1 = q.y, wz0 = 1.f - q.z, wz1 = q.z;
    w[0] = wx0 * wy0 * wz0; w[1] = wx0 * wy0 * wz1; w[2] = wx0 * wy1 * wz0; w[3] = wx0 * wy1 * wz1;
    w[4] = wx1 * wy0 * wz0; w[5] = wx1 * wy0 * wz1; w[6] = wx1 * wy1 * wz0; w[7] = wx1 * wy1 * wz1;
}
static inline real rinterp8(const real* g, const real* w) {
    real s = 0.f;
    for (int i = 0; i < 8; ++i) s += g[i] * w[i];
    return s;
}
static inline real rrnorm3(real x, real y, real z) { return (real)1 / SQRTR(x * x + y * y + z * z + (real)1e-15f); }

static void ray_of_pixel(int px, int py, int W, int H, float tanfovx, float tanfovy, float cx, float cy,
                         const float* c2w, r3* ro, r3* rd, r3* rd_inv, real* rd_norm_inv)
{
    real pfx = (real)px, pfy = (real)py;
    r3 cam_rd = rk((pfx + 0.5f - cx) * 2.f * tanfovx / (real)W, (pfy + 0.5f - cy) * 2.f * tanfovy / (real)H, 1.f);
    real rd_norm = SQRTR(rdot(cam_rd, cam_rd));
    r3 raw = rk(c2w[0] * cam_rd.x + c2w[1] * cam_rd.y + c2w[2] * cam_rd.z,
                c2w[4] * cam_rd.x + c2w[5] * cam_rd.y + c2w[6] * cam_rd.z,
                c2w[8] * cam_rd.x + c2w[9] * cam_rd.y + c2w[10] * cam_rd.z);
    *rd_norm_inv = (real)1 / rd_norm;
    *ro = rk(c2w[3], c2w[7], c2w[11]);
    *rd = rmuls(raw, *rd_norm_inv);
    *rd_inv = rk((real)1 / rd->x, (real)1 / rd->y, (real)1 / rd->z);
}

static inline int pix_in_bbox(int px, int py, uint32_t b0, uint32_t b1) {
    return px >= (int)(b0 >> 16) && py >= (int)(b0 & 0xFFFF) && px <= (int)(b1 >> 16) && py <= (int)(b1 & 0xFFFF);
}

static inline int ray_quadrant(r3 rd) { return ((rd.x < 0) << 2) | ((rd.y < 0) << 1) | (rd.z < 0); }

void svo_render_fwd(int W, int H, float tanfovx, float tanfovy, float cx, float cy,
                    const float* c2w, const float* bg, int n_samp, int need_depth, int need_normal,
                    const uint32_t* ranges, const uint32_t* vals, const uint32_t* bboxes,
                    const real* centers, const real* lengths, const real* geos, const real* rgbs,
                    real s_val,
                    real* out_color, real* out_depth, real* out_normal, real* out_T,
                    real* max_w /* may be NULL */, uint32_t* tile_last, uint32_t* n_contrib)
{
    const int gx = (W + TILE - 1) / TILE, gy = (H + TILE - 1) / TILE;
    const int HW = H * W;
    /* max_w is a shared running maximum: keep that variant single-threaded */
    const int nth = max_w ? 1 : g_threads;
    #pragma omp parallel for schedule(dynamic, 4) num_threads(nth)
    for (int tile = 0; tile < gx * gy; ++tile) {
        const int ty = tile / gx, tx = tile % gx;
        const uint32_t r0 = ranges[2 * tile], r1 = ranges[2 * tile + 1];
        uint32_t tl = r0;
        for (int py = ty * TILE; py < ty * TILE + TILE && py < H; ++py)
        for (int px = tx * TILE; px < tx * TILE + TILE && px < W; ++px) {
            if (g_pixel_mask && !g_pixel_mask[py * W + px]) continue;
            r3 ro, rd, rd_inv; real rni;
            ray_of_pixel(px, py, W, H, tanfovx, tanfovy, cx, cy, c2w, &ro, &rd, &rd_inv, &rni);
            const int pq = ray_quadrant(rd);
            real T = 1.f, D = 0.f; r3 Cc = rk(0, 0, 0), Nn = rk(0, 0, 0);
            int med_vox = -1; real med_T = 0.f, D_med = 0.f;
            uint32_t last = 0;
            for (uint32_t k = r0; k < r1; ++k) {
                const uint32_t val = vals[k];
                const uint32_t vid = val & 0x1FFFFFFFu, q = val >> 29;
                if (!pix_in_bbox(px, py, bboxes[2 * vid], bboxes[2 * vid + 1]) || (uint32_t)pq != q) continue;
                r3 vc = rk(centers[3 * vid], centers[3 * vid + 1], centers[3 * vid + 2]);
                real vl = lengths[vid];
                real a, b;
                rray_aabb(vc, vl, ro, rd_inv, &a, &b);
                if (a > b) continue;
                const real* g = geos + 8 * (size_t)vid;
                real w[8], la[3] = {0, 0, 0};
                real vli = (real)1 / vl;
                r3 pe = radd(ro, rmuls(rd, a));
                r3 pstep = rk((b - a) * rd.x / n_samp, (b - a) * rd.y / n_samp, (b - a) * rd.z / n_samp);
                r3 qe = rmuls(rsub(pe, rsubs(vc, (real)0.5f * vl)), vli);
                r3 qs = rmuls(pstep, vli);
                rtri_w(qe, w);
                real sdf_f = rinterp8(g, w);
                real phi_f = (real)1 / ((real)1 + EXPR(-s_val * sdf_f));
                real phi_e = phi_f;
                for (int s = 0; s < n_samp; ++s) {
                    r3 qc = radd(qe, rmuls(qs, (real)(s + 1)));
                    rtri_w(qc, w);
                    real sdf_c = rinterp8(g, w);
                    real phi_c = (real)1 / ((real)1 + EXPR(-s_val * sdf_c));
                    if (need_depth && n_samp > 1) la[s] = rmax((phi_f - phi_c) / (phi_f + (real)1e-6f), 0.f);
                    phi_f = phi_c; sdf_f = sdf_c;
                }
                real alpha = rmax((phi_e - phi_f) / (phi_e + (real)1e-6f), 0.f);
                if (g_trace && dabs((double)alpha - (double)MIN_ALPHA) <= TR_ALPHA_BAND) g_trace[py * W + px] |= TR_ALPHA;
                if (alpha < MIN_ALPHA) continue;
                if (g_trace && need_depth && dabs((double)T - 0.5) <= TR_MED_BAND) g_trace[py * W + px] |= TR_MEDIAN;
                real pw = T * alpha;
                Cc = radd(Cc, rmuls(rk(rgbs[3 * vid], rgbs[3 * vid + 1], rgbs[3 * vid + 2]), pw));
                if (need_depth) {
                    real dval;
                    if (n_samp == 3) {
                        real st = (real)0.3333333f * (b - a);
                        real t0 = a + (real)0.5f * st, t1 = a + (real)1.5f * st, t2 = a + (real)2.5f * st;
                        dval = la[0] * t0 + (1.f - la[0]) * la[1] * t1 + (1.f - la[0]) * (1.f - la[1]) * la[2] * t2;
                    } else if (n_samp == 2) {
                        real st = (real)0.5f * (b - a);
                        real t0 = a + (real)0.5f * st, t1 = a + (real)1.5f * st;
                        dval = la[0] * t0 + (1.f - la[0]) * la[1] * t1;
                    } else {
                        dval = alpha * (real)0.5f * (a + b);
                    }
                    D = D + T * dval;
                    if (T > 0.5f) { med_vox = (int)vid; med_T = T; }
                }
                if (need_normal) {
                    real nx = (g[4] + g[5] + g[6] + g[7]) - (g[0] + g[1] + g[2] + g[3]);
                    real ny = (g[2] + g[3] + g[6] + g[7]) - (g[0] + g[1] + g[4] + g[5]);
                    real nz = (g[1] + g[3] + g[5] + g[7]) - (g[0] + g[2] + g[4] + g[6]);
                    real rl = rrnorm3(nx, ny, nz);
                    Nn = radd(Nn, rmuls(rk(nx, ny, nz), pw * rl));
                }
                T *= (1.f - alpha);
                if (g_trace && dabs((double)T - (double)EARLY_STOP_T) <= TR_STOP_BAND) g_trace[py * W + px] |= TR_STOP;
                last = k - r0 + 1;
                if (max_w && pw > max_w[vid]) max_w[vid] = pw;
                if (T < EARLY_STOP_T) break;
            }
            if (need_depth && med_vox != -1) {
                /* forward.cu:450-521, SDF branch */
                r3 vc = rk(centers[3 * med_vox], centers[3 * med_vox + 1], centers[3 * med_vox + 2]);
                real vl = lengths[med_vox];
                const real* g = geos + 8 * (size_t)med_vox;
                real a, b;
                rray_aabb(vc, vl, ro, rd_inv, &a, &b);
                real vli = (real)1 / vl;
                real st = (b - a) * ((real)1.f / 16);
                r3 step = rmuls(rd, st);
                D_med = a - (real)0.5f * st;
                r3 qe = rmuls(rsub(radd(ro, rmuls(rd, a)), rsubs(vc, (real)0.5f * vl)), vli);
                r3 qs = rmuls(step, vli);
                real w[8];
                rtri_w(qe, w);
                real phi_p = (real)1 / ((real)1 + EXPR(-s_val * rinterp8(g, w)));
                for (int s = 0; s < 16 && med_T > 0.5f; ++s) {
                    D_med += st;
                    qe = radd(qe, qs);
                    rtri_w(qe, w);
                    real phi_c = (real)1 / ((real)1 + EXPR(-s_val * rinterp8(g, w)));
                    real ak = (phi_p - phi_c) / (phi_p + (real)1e-6f);
                    med_T *= (1.f - ak);
                    if (g_trace && dabs((double)med_T - 0.5) <= TR_MED_BAND) g_trace[py * W + px] |= TR_MEDIAN;
                    phi_p = phi_c;
                }
            }
            const int pid = py * W + px;
            n_contrib[pid] = last;
            out_color[pid] = Cc.x + T * bg[0];
            out_color[HW + pid] = Cc.y + T * bg[1];
            out_color[2 * HW + pid] = Cc.z + T * bg[2];
            out_T[pid] = T;
            if (need_depth) {
                out_depth[pid] = D * rni;
                out_depth[HW + pid] = 0.f;
                out_depth[2 * HW + pid] = D_med * rni;
                out_depth[3 * HW + pid] = 0.f;
            }
            if (need_normal) {
                out_normal[pid] = Nn.x; out_normal[HW + pid] = Nn.y; out_normal[2 * HW + pid] = Nn.z;
            }
            if (r0 + last > tl) tl = r0 + last;
        }
        tile_last[tile] = tl;
    }
}

/* ------------------------------------------------------------------ render backward
 * cuda/src/backward.cu:41-851 instantiated as the reference dispatches SDF mode
 * (always n_samp = 3, backward.cu:944-946), no distortion, lambda_ascending = 0.
 * dL_dvox[N,12] = [8 corner sdf | 3 rgb | |dL/dalpha * alpha|]; dL_ds scalar. */
void svo_render_bwd(int W, int H, float tanfovx, float tanfovy, float cx, float cy,
                    const float* c2w, const float* bg, int need_depth, int need_normal,
                    const uint32_t* ranges, const uint32_t* tile_last, const uint32_t* vals,
                    const uint32_t* bboxes, const real* centers, const real* lengths,
                    const real* geos, const real* rgbs, real s_val,
                    const real* out_T, const uint32_t* n_contrib,
                    const real* dL_dcolor, const real* dL_ddepth, const real* dL_dnormal,
                    const real* dL_dT, real lambda_R_concen, const real* gt_color,
                    real* dL_dvox, real* dL_ds)
{
    const int gx = (W + TILE - 1) / TILE, gy = (H + TILE - 1) / TILE;
    const int HW = H * W;
    const real WH_inv = (real)1 / ((real)(W * H));
    const real wR = lambda_R_concen * WH_inv;
    double ds_acc = 0.0;
    const int nth = g_threads;
    #pragma omp parallel for schedule(dynamic, 4) num_threads(nth) reduction(+ : ds_acc)
    for (int tile = 0; tile < gx * gy; ++tile) {
        const int ty = tile / gx, tx = tile % gx;
        const uint32_t r0 = ranges[2 * tile], r1 = tile_last[tile];
        for (int py = ty * TILE; py < ty * TILE + TILE && py < H; ++py)
        for (int px = tx * TILE; px < tx * TILE + TILE && px < W; ++px) {
            if (g_pixel_mask && !g_pixel_mask[py * W + px]) continue;
            r3 ro, rd, rd_inv; real rni;
            ray_of_pixel(px, py, W, H, tanfovx, tanfovy, cx, cy, c2w, &ro, &rd, &rd_inv, &rni);
            const int pq = ray_quadrant(rd);
            const int pid = py * W + px;
            real T = out_T[pid];
            const uint32_t lastc = n_contrib[pid];
            r3 dpix = rk(dL_dcolor[pid], dL_dcolor[HW + pid], dL_dcolor[2 * HW + pid]);
            real last_dT = dL_dT[pid] + rdot(rk(bg[0], bg[1], bg[2]), dpix);
            real dD = need_depth ? dL_ddepth[pid] * rni : 0.f;
            r3 dN = need_normal ? rk(dL_dnormal[pid], dL_dnormal[HW + pid], dL_dnormal[2 * HW + pid]) : rk(0, 0, 0);
            r3 gt = rk(0, 0, 0);
            if (lambda_R_concen > 0) gt = rk(gt_color[pid], gt_color[HW + pid], gt_color[2 * HW + pid]);
            for (int64_t k = (int64_t)r1 - 1; k >= (int64_t)r0; --k) {
                if ((uint32_t)(k - r0) >= lastc) continue;
                const uint32_t val = vals[k];
                const uint32_t vid = val & 0x1FFFFFFFu, q = val >> 29;
                if (!pix_in_bbox(px, py, bboxes[2 * vid], bboxes[2 * vid + 1]) || (uint32_t)pq != q) continue;
                r3 vc = rk(centers[3 * vid], centers[3 * vid + 1], centers[3 * vid + 2]);
                real vl = lengths[vid];
                real a, b;
                rray_aabb(vc, vl, ro, rd_inv, &a, &b);
                if (a > b) continue;
                const real* g = geos + 8 * (size_t)vid;
                real vli = (real)1 / vl;
                real dg[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                real we[8], wx[8];
                /* backward.cu:313-337 entry / exit from ro + t rd */
                r3 pe = radd(ro, rmuls(rd, a)), px_ = radd(ro, rmuls(rd, b));
                r3 lo = rsubs(vc, (real)0.5f * vl);
                r3 qe = rmuls(rsub(pe, lo), vli), qx = rmuls(rsub(px_, lo), vli);
                rtri_w(qe, we); rtri_w(qx, wx);
                real sdf_e = 0.f, sdf_x = 0.f;
                for (int i = 0; i < 8; ++i) { sdf_e += g[i] * we[i]; sdf_x += g[i] * wx[i]; }
                real phi_e = (real)1 / ((real)1 + EXPR(-s_val * sdf_e));
                real phi_x = (real)1 / ((real)1 + EXPR(-s_val * sdf_x));
                real denom = phi_e + (real)1e-6f;
                real alpha = rmax((phi_e - phi_x) / denom, 0.f);
                real la[3] = {0, 0, 0};
                real eg[3][8];
                memset(eg, 0, sizeof(eg));
                if (need_depth) {
                    /* backward.cu:338-388 */
                    r3 q0 = rmuls(rsub(radd(ro, rmuls(rd, a)), lo), vli);
                    r3 qst = rk((b - a) * rd.x / 3 * vli, (b - a) * rd.y / 3 * vli, (b - a) * rd.z / 3 * vli);
                    for (int s = 0; s < 3; ++s) {
                        r3 qk = radd(q0, rmuls(qst, (real)s)), qk1 = radd(q0, rmuls(qst, (real)(s + 1)));
                        real wk[8], wk1[8];
                        rtri_w(qk, wk); rtri_w(qk1, wk1);
                        real sk = 0.f, sk1 = 0.f;
                        for (int i = 0; i < 8; ++i) { sk += g[i] * wk[i]; sk1 += g[i] * wk1[i]; }
                        real pk = (real)1 / ((real)1 + EXPR(-s_val * sk));
                        real pk1 = (real)1 / ((real)1 + EXPR(-s_val * sk1));
                        real dk = pk + (real)1e-6f;
                        real raw = (pk - pk1) / dk;
                        real allow = raw > 0.f ? 1.f : 0.f;
                        if (g_trace && dabs((double)raw) <= TR_RAW_BAND && !(alpha < MIN_ALPHA)) g_trace[pid] |= TR_ADJ;
                        la[s] = rmax(raw, 0.f);
                        real d0 = allow * (pk1 / (dk * dk));
                        real d1 = allow * (-(real)1 / dk);
                        real p0 = s_val * pk * (1.f - pk);
                        real p1 = s_val * pk1 * (1.f - pk1);
                        for (int i = 0; i < 8; ++i) eg[s][i] += d0 * p0 * wk[i] + d1 * p1 * wk1[i];
                    }
                }
                if (g_trace && dabs((double)alpha - (double)MIN_ALPHA) <= TR_ALPHA_BAND) g_trace[pid] |= TR_ADJ;
                if (alpha < MIN_ALPHA) continue;   /* lambda_ascending = 0 */
                if (g_vox_trace && g_trace && (g_trace[pid] & (TR_ALPHA | TR_STOP | TR_MEDIAN))) g_vox_trace[vid] = 1;
                T = T / (1.f - alpha);
                real pw = alpha * T;
                r3 c = rk(rgbs[3 * vid], rgbs[3 * vid + 1], rgbs[3 * vid + 2]);
                real dpw = rdot(dpix, c);
                if (need_normal) {
                    /* backward.cu:604-639 */
                    real nx = (g[4] + g[5] + g[6] + g[7]) - (g[0] + g[1] + g[2] + g[3]);
                    real ny = (g[2] + g[3] + g[6] + g[7]) - (g[0] + g[1] + g[4] + g[5]);
                    real nz = (g[1] + g[3] + g[5] + g[7]) - (g[0] + g[2] + g[4] + g[6]);
                    r3 ln = rk(nx, ny, nz);
                    real rl = rrnorm3(nx, ny, nz);
                    r3 sn = rmuls(ln, rl);
                    dpw += rdot(dN, sn);
                    r3 dsn = rmuls(dN, pw);
                    real t = rdot(dsn, ln) * rl;
                    r3 dln = rmuls(rsub(dsn, rmuls(sn, t)), rl);
                    dg[0] += -dln.x - dln.y - dln.z; dg[1] += -dln.x - dln.y + dln.z;
                    dg[2] += -dln.x + dln.y - dln.z; dg[3] += -dln.x + dln.y + dln.z;
                    dg[4] += +dln.x - dln.y - dln.z; dg[5] += +dln.x - dln.y + dln.z;
                    dg[6] += +dln.x + dln.y - dln.z; dg[7] += +dln.x + dln.y + dln.z;
                }
                real dalpha = T * (dpw - last_dT);
                last_dT += alpha * (dpw - last_dT);
                {
                    /* backward.cu:650-671 */
                    real ppe = s_val * phi_e * (1.f - phi_e);
                    real ppx = s_val * phi_x * (1.f - phi_x);
                    real dae = (ppe * (1.f - alpha)) / denom;
                    real dax = -ppx / denom;
                    for (int i = 0; i < 8; ++i) {
                        dg[i] += dae * we[i] * dalpha;
                        dg[i] += dax * wx[i] * dalpha;
                    }
                    real dpe = phi_e * (1.f - phi_e) * sdf_e;
                    real dpx = phi_x * (1.f - phi_x) * sdf_x;
                    real das = ((dpe * (1.f - alpha)) + (-dpx)) / denom;
                    ds_acc += (double)(dalpha * das);
                }
                if (need_depth) {
                    /* backward.cu:682-768, n_samp = 3, SDF */
                    real st = (real)0.3333333f * (b - a);
                    real a0 = la[0], a1 = la[1], a2 = la[2];
                    real t0 = a + (real)0.5f * st, t1 = a + (real)1.5f * st, t2 = a + (real)2.5f * st;
                    real dval = a0 * t0 + (1.f - a0) * a1 * t1 + (1.f - a0) * (1.f - a1) * a2 * t2;
                    real d0 = dD * T * (t0 + a1 * a2 * t2 - a1 * t1 - a2 * t2);
                    real d1 = dD * T * (t1 + a0 * a2 * t2 - a0 * t1 - a2 * t2);
                    real d2 = dD * T * (t2 + a0 * a1 * t2 - a0 * t2 - a1 * t2);
                    last_dT += dD * dval;
                    for (int i = 0; i < 8; ++i) dg[i] += d0 * eg[0][i] + d1 * eg[1][i] + d2 * eg[2][i];
                }
                real drgb[3] = {pw * dpix.x, pw * dpix.y, pw * dpix.z};
                if (lambda_R_concen > 0) {
                    drgb[0] += wR * pw * 2.0f * (c.x - gt.x);
                    drgb[1] += wR * pw * 2.0f * (c.y - gt.y);
                    drgb[2] += wR * pw * 2.0f * (c.z - gt.z);
                }
                real* o = dL_dvox + 12 * (size_t)vid;
                real pack[12];
                for (int i = 0; i < 8; ++i) pack[i] = dg[i];
                pack[8] = drgb[0]; pack[9] = drgb[1]; pack[10] = drgb[2];
                pack[11] = FABSR(dalpha * alpha);
                real* oa = g_abs_sum ? (real*)g_abs_sum + 12 * (size_t)vid : NULL;
                if (nth == 1) {
                    for (int i = 0; i < 12; ++i) o[i] += pack[i];
                    if (oa) for (int i = 0; i < 12; ++i) oa[i] += FABSR(pack[i]);
                } else {
                    for (int i = 0; i < 12; ++i) {
                        #pragma omp atomic update
                        o[i] += pack[i];
                    }
                    if (oa) for (int i = 0; i < 12; ++i) {
                        #pragma omp atomic update
                        oa[i] += FABSR(pack[i]);
                    }
                }
            }
        }
    }
    *dL_ds = (real)ds_acc;
}

/* ------------------------------------------------------------------ gather
 * cuda/src/geo_params_gather.cu:22-72 */
void svo_gather_geo(int n_care, const int64_t* care_idx, const int64_t* vox_key, const float* grid, float* geos) {
    for (int t = 0; t < n_care; ++t) {
        int64_t i = care_idx[t];
        for (int k = 0; k < 8; ++k) geos[8 * i + k] = grid[vox_key[8 * i + k]];
    }
}
void svo_gather_geo_bw(int n_care, const int64_t* care_idx, const int64_t* vox_key, const float* dgeos, float* dgrid) {
    for (int t = 0; t < n_care; ++t) {
        int64_t i = care_idx[t];
        for (int k = 0; k < 8; ++k) dgrid[vox_key[8 * i + k]] += dgeos[8 * i + k];
    }
}

/* ------------------------------------------------------------------ SH
 * cuda/src/sh_compute.cu:33-176 */
static const float C0 = 0.28209479177387814f, C1 = 0.4886025119029199f;
static const float C2[5] = {1.0925484305920792f, -1.0925484305920792f, 0.31539156525252005f,
                            -1.0925484305920792f, 0.5462742152960396f};
static const float C3[7] = {-0.5900435899266435f, 2.890611442640554f, -0.4570457994644658f,
                            0.3731763325901154f, -0.4570457994644658f, 1.445305721320277f,
                            -0.5900435899266435f};

static void sh_basis(int deg, f3 dir, float* basis /* 16 */) {
    float x = dir.x, y = dir.y, z = dir.z;
    basis[0] = C0;
    if (deg > 0) { basis[1] = -C1 * y; basis[2] = C1 * z; basis[3] = -C1 * x; }
    if (deg > 1) {
        float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
        basis[4] = C2[0] * xy; basis[5] = C2[1] * yz; basis[6] = C2[2] * (2.0f * zz - xx - yy);
        basis[7] = C2[3] * xz; basis[8] = C2[4] * (xx - yy);
        if (deg > 2) {
            basis[9] = C3[0] * y * (3.0f * xx - yy); basis[10] = C3[1] * xy * z;
            basis[11] = C3[2] * y * (4.0f * zz - xx - yy); basis[12] = C3[3] * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
            basis[13] = C3[4] * x * (4.0f * zz - xx - yy); basis[14] = C3[5] * z * (xx - yy);
            basis[15] = C3[6] * x * (xx - 3.0f * yy);
        }
    }
}

void svo_sh_eval(int N, int n_idx, const int64_t* idx, int deg, int M /* coeffs incl. dc */,
                 const float* centers, const float* cam_pos, const float* sh0, const float* shs, float* rgbs)
{
    int n = n_idx > 0 ? n_idx : N;
    memset(rgbs, 0, sizeof(float) * 3 * (size_t)N);
    for (int t = 0; t < n; ++t) {
        int64_t i = n_idx > 0 ? idx[t] : t;
        f3 d = mk(centers[3 * i] - cam_pos[0], centers[3 * i + 1] - cam_pos[1], centers[3 * i + 2] - cam_pos[2]);
        float r = 1.f / sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
        d = muls(d, r);
        float basis[16];
        sh_basis(deg, d, basis);
        int nb = (deg + 1) * (deg + 1);
        for (int c = 0; c < 3; ++c) {
            float v = basis[0] * sh0[3 * i + c];
            for (int k = 1; k < nb; ++k) v += basis[k] * shs[((size_t)i * (M - 1) + (k - 1)) * 3 + c];
            v += 0.5f;
            rgbs[3 * i + c] = v * (float)(v > 0.0f);   /* sh_compute.cu:102-104 */
        }
    }
}

void svo_sh_eval_bw(int N, int n_idx, const int64_t* idx, int deg, int M, const float* centers,
                    const float* cam_pos, const float* drgbs, float* dsh0, float* dshs)
{
    int n = n_idx > 0 ? n_idx : N;
    memset(dsh0, 0, sizeof(float) * 3 * (size_t)N);
    memset(dshs, 0, sizeof(float) * 3 * (size_t)N * (M - 1));
    for (int t = 0; t < n; ++t) {
        int64_t i = n_idx > 0 ? idx[t] : t;
        f3 d = mk(centers[3 * i] - cam_pos[0], centers[3 * i + 1] - cam_pos[1], centers[3 * i + 2] - cam_pos[2]);
        float r = 1.f / sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
        d = muls(d, r);
        float basis[16];
        sh_basis(deg, d, basis);
        int nb = (deg + 1) * (deg + 1);
        for (int c = 0; c < 3; ++c) {
            dsh0[3 * i + c] = basis[0] * drgbs[3 * i + c];
            for (int k = 1; k < nb; ++k) dshs[((size_t)i * (M - 1) + (k - 1)) * 3 + c] = basis[k] * drgbs[3 * i + c];
        }
    }
}

/* ------------------------------------------------------------------ valid gradient table
 * cuda/src/utils.cu:190-252 + the key sort of src/utils/octree_utils.py:293-314. */
static int valid_cells(const float* c, float size, const float* sc, float ext, int res, int leaf, int* lo, int* hi) {
    float cells = (size / ext) * res;
    if (!leaf && (cells > 1.5f || cells < 0.9f)) return 0;
    if (leaf && cells < 0.9f) return 0;
    float mn[3], mx[3];
    for (int d = 0; d < 3; ++d) { mn[d] = sc[d] - 0.5f * ext; mx[d] = sc[d] + 0.5f * ext; }
    for (int d = 0; d < 3; ++d) if (c[d] < mn[d] || c[d] > mx[d]) return 0;
    for (int d = 0; d < 3; ++d) {
        float a = c[d] - 0.5f * size, b = c[d] + 0.5f * size;
        lo[d] = (int)roundf((a - mn[d]) / (mx[d] - mn[d]) * res);
        hi[d] = (int)roundf((b - mn[d]) / (mx[d] - mn[d]) * res);
        /* clamp to the grid; the reference writes past grid_mask in this case */
        lo[d] = lo[d] < 0 ? 0 : (lo[d] > res ? res : lo[d]);
        hi[d] = hi[d] < 0 ? 0 : (hi[d] > res ? res : hi[d]);
    }
    return 1;
}

int64_t svo_valid_table_count(int N, const float* centers, const float* sizes, const float* sc, float ext,
                              int res_pow2, const uint8_t* is_leaf) {
    int res = 1 << res_pow2; int64_t n = 0;
    for (int i = 0; i < N; ++i) {
        int lo[3], hi[3];
        if (!valid_cells(centers + 3 * i, sizes[i], sc, ext, res, is_leaf[i], lo, hi)) continue;
        int64_t a = hi[0] - lo[0], b = hi[1] - lo[1], c = hi[2] - lo[2];
        if (a > 0 && b > 0 && c > 0) n += a * b * c;
    }
    return n;
}

typedef struct { int32_t key; int32_t vox; } kv_t;
static int cmp_kv(const void* a, const void* b) {
    const kv_t* x = (const kv_t*)a; const kv_t* y = (const kv_t*)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->vox < y->vox ? -1 : (x->vox > y->vox);
}

void svo_valid_table(int N, const float* centers, const float* sizes, const float* sc, float ext, int res_pow2,
                     const uint8_t* is_leaf, uint8_t* grid_mask, int32_t* keys, int32_t* g2v) {
    int res = 1 << res_pow2; int64_t n = 0;
    memset(grid_mask, 0, (size_t)res * res * res);
    int64_t total = svo_valid_table_count(N, centers, sizes, sc, ext, res_pow2, is_leaf);
    kv_t* kv = (kv_t*)malloc(sizeof(kv_t) * (total > 0 ? total : 1));
    for (int i = 0; i < N; ++i) {
        int lo[3], hi[3];
        if (!valid_cells(centers + 3 * i, sizes[i], sc, ext, res, is_leaf[i], lo, hi)) continue;
        for (int x = lo[0]; x < hi[0]; ++x) for (int y = lo[1]; y < hi[1]; ++y) for (int z = lo[2]; z < hi[2]; ++z) {
            int f = x + res * (y + res * z);
            grid_mask[f] = 1; kv[n].key = f; kv[n].vox = i; n++;
        }
    }
    qsort(kv, (size_t)n, sizeof(kv_t), cmp_kv);
    for (int64_t k = 0; k < n; ++k) { keys[k] = kv[k].key; g2v[k] = kv[k].vox; }
    free(kv);
}

/* ------------------------------------------------------------------ smoothness losses
 * cuda/src/auxiliary.h:392-454 (neighbour test, key search, clamped trilinear sample) and
 * the hash RNG of auxiliary.h:455-471; Laplacian cuda/src/ls_compute.cu:14-109, grid
 * Eikonal cuda/src/ge_compute.cu:14-117.  The reference seeds with clock64(); here the
 * seed is an argument. */
static float hash_to_float(uint32_t x) {
    x ^= x >> 17; x *= 0xed5ad4bbu; x ^= x >> 11; x *= 0xac4c1b51u; x ^= x >> 15; x *= 0x31848babu; x ^= x >> 14;
    return (float)(x & 0xFFFFFF) / (float)0x1000000;
}
static f3 rand_vec(int tid, int seed) {
    return mk(hash_to_float((uint32_t)((uint32_t)seed * 73856093u ^ (uint32_t)(tid * 3 + 0))),
              hash_to_float((uint32_t)((uint32_t)seed * 19349663u ^ (uint32_t)(tid * 3 + 1))),
              hash_to_float((uint32_t)((uint32_t)seed * 83492791u ^ (uint32_t)(tid * 3 + 2))));
}
static int bsearch_key(const int32_t* keys, int n, int key) {
    int l = 0, r = n - 1;
    while (l <= r) { int m = (l + r) / 2; if (keys[m] == key) return m; if (keys[m] < key) l = m + 1; else r = m - 1; }
    return -1;
}
static int nb_ok(int x, int y, int z, int res, const uint8_t* mask) {
    if (x <= 0 || x >= res - 1 || y <= 0 || y >= res - 1 || z <= 0 || z >= res - 1) return 0;
    #define F(a, b, c) ((a) + (b) * res + (c) * res * res)
    return mask[F(x + 1, y, z)] && mask[F(x - 1, y, z)] && mask[F(x, y + 1, z)] && mask[F(x, y - 1, z)] &&
           mask[F(x, y, z + 1)] && mask[F(x, y, z - 1)];
    #undef F
}
static float sample_sdf(int G, int x, int y, int z, const int32_t* keys, const int32_t* g2v, const float* coords,
                        const float* vsizes, const int64_t* vox_key, const float* grid, int res, f3 rv,
                        float* w, int* vid) {
    int gk = x + y * res + z * res * res;
    int id = bsearch_key(keys, G, gk);
    if (id < 0) { *vid = -1; return 0.f; }
    int v = g2v[id]; *vid = v;
    f3 pt = mk(x + rv.x, y + rv.y, z + rv.z);
    f3 base = mk(coords[3 * v], coords[3 * v + 1], coords[3 * v + 2]);
    float sz = vsizes[v];
    f3 lq = mk((pt.x - base.x) / sz, (pt.y - base.y) / sz, (pt.z - base.z) / sz);
    tri_w(lq, w);
    float s = 0.f;
    for (int i = 0; i < 8; ++i) { if (w[i] < 0) w[i] = 0; if (w[i] > 1) w[i] = 1; s += grid[vox_key[8 * v + i]] * w[i]; }
    return s;
}
static void scatter8(int v, const int64_t* vox_key, const float* w, float d, float* grad) {
    if (v < 0) return;
    for (int i = 0; i < 8; ++i) grad[vox_key[8 * v + i]] += d * w[i];
}

void svo_laplacian_bw(int G, int A, const int32_t* active, const int32_t* keys, const int32_t* g2v, int res,
                      const uint8_t* mask, const float* coords, const float* vsizes, const int64_t* vox_key,
                      const float* grid, float weight, float vox_size_inv, int seed, float* grad) {
    static const int dx[6] = {1, -1, 0, 0, 0, 0}, dy[6] = {0, 0, 1, -1, 0, 0}, dz[6] = {0, 0, 0, 0, 1, -1};
    for (int t = 0; t < A; ++t) {
        int gk = keys[active[t]];
        int x = gk % res, y = (gk / res) % res, z = gk / (res * res);
        if (!mask[gk] || !nb_ok(x, y, z, res, mask)) continue;
        f3 rv = rand_vec(t, seed);
        float w[7][8]; int vid[7]; float nb[6];
        float c = sample_sdf(G, x, y, z, keys, g2v, coords, vsizes, vox_key, grid, res, rv, w[0], &vid[0]);
        for (int i = 0; i < 6; ++i)
            nb[i] = sample_sdf(G, x + dx[i], y + dy[i], z + dz[i], keys, g2v, coords, vsizes, vox_key, grid, res, rv, w[i + 1], &vid[i + 1]);
        float lx = nb[0] + nb[1] - 2.0f * c, ly = nb[2] + nb[3] - 2.0f * c, lz = nb[4] + nb[5] - 2.0f * c;
        float lr = sqrtf(lx * lx + ly * ly + lz * lz + 1e-10f);
        /* ls_compute.cu:79-83 evaluates these in double (0.5 is a double literal) */
        float size = (float)((double)weight * 0.5 * (double)vox_size_inv * (double)vox_size_inv);
        float gx_ = (float)(0.5 / (double)lr * 2 * (double)lx * (double)size);
        float gy_ = (float)(0.5 / (double)lr * 2 * (double)ly * (double)size);
        float gz_ = (float)(0.5 / (double)lr * 2 * (double)lz * (double)size);
        float gc = -2.0f * (gx_ + gy_ + gz_);
        scatter8(vid[0], vox_key, w[0], gc, grad);
        scatter8(vid[1], vox_key, w[1], gx_, grad); scatter8(vid[2], vox_key, w[2], gx_, grad);
        scatter8(vid[3], vox_key, w[3], gy_, grad); scatter8(vid[4], vox_key, w[4], gy_, grad);
        scatter8(vid[5], vox_key, w[5], gz_, grad); scatter8(vid[6], vox_key, w[6], gz_, grad);
    }
}

void svo_eikonal_bw(int G, int A, const int32_t* active, const int32_t* keys, const int32_t* g2v, int res,
                    const uint8_t* mask, const float* coords, const float* vsizes, const int64_t* vox_key,
                    const float* grid, float weight, float vox_size_inv, int seed, float* grad) {
    static const int dx[6] = {1, -1, 0, 0, 0, 0}, dy[6] = {0, 0, 1, -1, 0, 0}, dz[6] = {0, 0, 0, 0, 1, -1};
    for (int t = 0; t < A; ++t) {
        int gk = keys[active[t]];
        int x = gk % res, y = (gk / res) % res, z = gk / (res * res);
        if (!mask[gk] || !nb_ok(x, y, z, res, mask)) continue;
        f3 rv = rand_vec(t, seed);
        float w[6][8]; int vid[6]; float s[6];
        for (int i = 0; i < 6; ++i)
            s[i] = sample_sdf(G, x + dx[i], y + dy[i], z + dz[i], keys, g2v, coords, vsizes, vox_key, grid, res, rv, w[i], &vid[i]);
        float dxv = (s[0] - s[1]) * 0.5f, dyv = (s[2] - s[3]) * 0.5f, dzv = (s[4] - s[5]) * 0.5f;
        float gn = sqrtf(dxv * dxv + dyv * dyv + dzv * dzv + 1e-6f);
        /* ge_compute.cu:93 evaluates grad_world in double (0.5 is a double literal) */
        float gw = (float)((double)gn * 0.5 * (double)vox_size_inv);
        float dg = 2.0f * (gw - 1.0f) * weight;
        float ddx = dg * dxv / gn * 0.5f * vox_size_inv;
        float ddy = dg * dyv / gn * 0.5f * vox_size_inv;
        float ddz = dg * dzv / gn * 0.5f * vox_size_inv;
        scatter8(vid[0], vox_key, w[0], ddx, grad); scatter8(vid[1], vox_key, w[1], -ddx, grad);
        scatter8(vid[2], vox_key, w[2], ddy, grad); scatter8(vid[3], vox_key, w[3], -ddy, grad);
        scatter8(vid[4], vox_key, w[4], ddz, grad); scatter8(vid[5], vox_key, w[5], -ddz, grad);
    }
}

/* ------------------------------------------------------------------ other grid regularisers
 * Voxel Eikonal, cuda/src/vg_compute.cu:23-77: per active voxel the centre gradient from its
 * 8 corners (sign of bit 2 / 1 / 0 for x / y / z), loss gradient 4 (|g|^2 - 2) w g, chained
 * to the corners with the factor 0.25. */
void svo_voxel_gradient_bw(int A, const int32_t* active, const int64_t* vox_key, const float* grid,
                           const float* vox_size_inv, float weight, float* grad) {
    for (int t = 0; t < A; ++t) {
        int v = active[t];
        float inv4h = 0.25f * vox_size_inv[v];
        float S[8], gx = 0.f, gy = 0.f, gz = 0.f;
        for (int i = 0; i < 8; ++i) S[i] = grid[vox_key[8 * (int64_t)v + i]];
        for (int i = 0; i < 8; ++i) {
            float sx = (i & 4) ? 1.f : -1.f, sy = (i & 2) ? 1.f : -1.f, sz = (i & 1) ? 1.f : -1.f;
            gx += sx * S[i]; gy += sy * S[i]; gz += sz * S[i];
        }
        gx *= inv4h; gy *= inv4h; gz *= inv4h;
        float g2 = gx * gx + gy * gy + gz * gz;
        float sc = 4.f * (g2 - 2.f) * weight;
        float dx = sc * gx, dy = sc * gy, dz = sc * gz;
        for (int i = 0; i < 8; ++i) {
            float sx = (i & 4) ? 1.f : -1.f, sy = (i & 2) ? 1.f : -1.f, sz = (i & 1) ? 1.f : -1.f;
            grad[vox_key[8 * (int64_t)v + i]] += (dx * sx + dy * sy + dz * sz) * 0.25f;
        }
    }
}

/* Sign total variation, cuda/src/tv_compute.cu:22-158: per (voxel, channel) each corner gets
 * w * (sum over its 3 edge neighbours of +1 if it is larger, else -1), w = weight, times
 * 0.01 * vox_size_inv[voxel] unless no_tv_s.  With tv_sparse a (voxel, channel) takes part only
 * if one of its corners has a nonzero gradient; the reference tests that while other threads
 * add to the same gradient, so its outcome depends on timing.  Here the test reads the gradient
 * as it was on entry (a snapshot), the deterministic form of the same rule. */
void svo_total_variation_bw(int64_t N, int C, const int64_t* vox_key, const float* grid, float weight,
                            const float* vox_size_inv, int no_tv_s, int tv_sparse, float* grad, int64_t M) {
    float* snap = NULL;
    if (tv_sparse) {
        snap = (float*)malloc(sizeof(float) * (size_t)(M * C > 0 ? M * C : 1));
        memcpy(snap, grad, sizeof(float) * (size_t)(M * C));
    }
    for (int64_t n = 0; n < N; ++n) for (int c = 0; c < C; ++c) {
        const int64_t* k = vox_key + 8 * n;
        if (tv_sparse) {
            int valid = 0;
            for (int i = 0; i < 8; ++i) valid |= snap[k[i] * C + c] != 0.f;
            if (!valid) continue;
        }
        float v[8];
        for (int i = 0; i < 8; ++i) v[i] = grid[k[i] * C + c];
        float w = weight;
        if (!no_tv_s) w *= 0.01f * vox_size_inv[n];
        for (int i = 0; i < 8; ++i) {
            int s = ((v[i] > v[i ^ 1]) * 2 - 1) + ((v[i] > v[i ^ 2]) * 2 - 1) + ((v[i] > v[i ^ 4]) * 2 - 1);
            grad[k[i] * C + c] += w * (float)s;
        }
    }
    free(snap);
}

/* Points on the surface, cuda/src/pl_compute.cu:14-63: each point (grid units) is placed in
 * its cell by truncating casts, the owner voxel's trilinear SDF (weights not clamped, as in
 * auxiliary.h:319-333) is driven to zero, dL/dsdf = 2 sdf weight spread over the 8 corners.
 * A masked cell missing from the key table is skipped (the reference would read
 * grid2voxel[-1]). */
void svo_points_loss_bw(int P, const float* pts, int G, const int32_t* keys, const int32_t* g2v, int res,
                        const uint8_t* mask, const float* coords, const float* vsizes, const int64_t* vox_key,
                        const float* grid, float weight, float* grad) {
    for (int t = 0; t < P; ++t) {
        float px = pts[3 * t], py = pts[3 * t + 1], pz = pts[3 * t + 2];
        int ix = (int)px, iy = (int)py, iz = (int)pz;
        if (ix < 0 || ix >= res || iy < 0 || iy >= res || iz < 0 || iz >= res) continue;
        int key = ix + iy * res + iz * res * res;
        if (!mask[key]) continue;
        int id = bsearch_key(keys, G, key);
        if (id < 0) continue;
        int v = g2v[id];
        float sz = vsizes[v], w[8];
        tri_w(mk((px - coords[3 * v]) / sz, (py - coords[3 * v + 1]) / sz, (pz - coords[3 * v + 2]) / sz), w);
        float sdf = 0.f;
        for (int i = 0; i < 8; ++i) sdf += w[i] * grid[vox_key[8 * (int64_t)v + i]];
        float dL = 2.0f * (sdf - 0.0f) * weight;
        for (int i = 0; i < 8; ++i) grad[vox_key[8 * (int64_t)v + i]] += dL * w[i];
    }
}

/* ------------------------------------------------------------------ 8-bit checkpoint codebook
 * src/sparse_voxel_gears/io.py:123-167 (quantization): codebook initialised at the 257
 * quantiles (float32 positions j/256 * (n-1), truncated) with entry 0 set to -inf, a left
 * searchsorted, the nearer of the two candidate entries, then up to max_iter rounds of
 * (per-entry mean, move each value one entry towards a nearer neighbour), a final mean.
 * Index -1 reads entry 255 (torch's negative index), means are float sums in value order
 * divided by the count, entries with no values stay 0.  Returns the rounds that moved
 * values. */
static int cmp_f32(const void* a, const void* b) {
    float x = *(const float*)a, y = *(const float*)b;
    return (x > y) - (x < y);
}
static void quant_mean(int64_t n, const float* v, const int32_t* ind, float* cb) {
    float sum[256], cnt[256];
    for (int b = 0; b < 256; ++b) { sum[b] = 0.f; cnt[b] = 0.f; }
    for (int64_t i = 0; i < n; ++i) { sum[ind[i]] += v[i]; cnt[ind[i]] += 1.f; }
    for (int b = 0; b < 256; ++b) cb[b] = cnt[b] > 0.f ? sum[b] / cnt[b] : 0.f;
}
static inline int quant_moves(float x, const float* book, int k, int* dir) {
    float dl = fabsf(x - book[k - 1 < 0 ? 255 : k - 1]);
    float dr = fabsf(x - book[k + 1 > 255 ? 255 : k + 1]);
    float dm = fabsf(x - book[k]);
    *dir = (dr < dl) ? 1 : -1;
    return fminf(dl, dr) < dm;
}
int svo_quantize(int64_t n, const float* v, int max_iter, uint8_t* index_out, float* codebook_out) {
    if (n <= 0) return -1;
    float* sorted = (float*)malloc(sizeof(float) * (size_t)n);
    int32_t* ind = (int32_t*)calloc((size_t)n, sizeof(int32_t));
    memcpy(sorted, v, sizeof(float) * (size_t)n);
    qsort(sorted, (size_t)n, sizeof(float), cmp_f32);
    float full[257];
    for (int j = 0; j < 257; ++j) {
        volatile float pos = ((float)j / 256.0f) * (float)(n - 1);
        int64_t q = (int64_t)pos;
        if (q < 0) q = 0;
        if (q > n - 1) q = n - 1;
        full[j] = sorted[q];
    }
    full[0] = -INFINITY;
    const float* cb = full + 1;
    for (int64_t i = 0; i < n; ++i) {
        int lo = 0, hi = 257;                       /* first entry >= v (searchsorted, left) */
        while (lo < hi) { int mid = (lo + hi) / 2; if (full[mid] < v[i]) lo = mid + 1; else hi = mid; }
        int k = lo - 1;
        if (k < 0) k = 0;
        if (k > 255) k = 255;
        float dl = fabsf(v[i] - cb[k - 1 < 0 ? 255 : k - 1]), dm = fabsf(v[i] - cb[k]);
        k = k - 1 + (dm < dl);
        if (k < 0) k = 0;
        if (k > 255) k = 255;
        ind[i] = k;
    }
    float book[256];
    int rounds = 0, dir = 0;
    for (int it = 0; it < max_iter; ++it) {
        quant_mean(n, v, ind, book);
        int64_t moved = 0;
        for (int64_t i = 0; i < n; ++i) moved += quant_moves(v[i], book, ind[i], &dir);
        if (moved == 0) break;
        for (int64_t i = 0; i < n; ++i) {
            if (!quant_moves(v[i], book, ind[i], &dir)) continue;
            int k = ind[i] + dir;
            ind[i] = k < 0 ? 0 : (k > 255 ? 255 : k);
        }
        rounds++;
    }
    quant_mean(n, v, ind, codebook_out);
    for (int64_t i = 0; i < n; ++i) index_out[i] = (uint8_t)ind[i];
    free(sorted); free(ind);
    return rounds;
}

/* ------------------------------------------------------------------ normal-from-depth losses
 * src/cameras.py:104-127 (depth2pts: position + rd * depth, rd of cuda/src/utils.cu:47-72;
 * depth2normal: normalize(cross(dx, dy)) on the interior, dx / dy the differences of the points
 * pad = ks/2 to either side, optionally zeroed where dot(normal, normalize(pts - position)) <=
 * tol_cos) and src/utils/loss_utils.py:345-407: NormalDepthConsistencyLoss (alpha = 1 - T,
 * N = -normal * alpha, loss = mean((alpha^2 - <n_r, N>) * mask)) and
 * NormalMedianConsistencyLoss (N = -normal, loss = mean((1 - <n_r, N>) * mask)), mask = N != 0
 * anywhere.  Returns the loss (weight 1) and ADDS its gradient with respect to the depth plane
 * and the rendered normals (alpha, the tolerance mask and the loss mask held constant, as the
 * reference's no_grad / detach make them). */
double svo_normal_depth_loss(int W, int H, float cx, float cy, float tanfovx, float tanfovy, const float* c2w,
                             const float* depth, const float* nr, const float* T, int ks, float tol_cos,
                             float* grad_depth, float* grad_normal) {
    const int pad = ks / 2;
    const int64_t P = (int64_t)W * H;
    float* rd = (float*)malloc(sizeof(float) * 3 * P);
    float* pts = (float*)malloc(sizeof(float) * 3 * P);
    float* gdx = (float*)calloc((size_t)(3 * P), sizeof(float));
    float* gdy = (float*)calloc((size_t)(3 * P), sizeof(float));
    for (int y = 0; y < H; ++y) for (int x = 0; x < W; ++x) {
        int64_t q = (int64_t)y * W + x;
        float u = ((float)x + 0.5f - cx) * 2.f * tanfovx / (float)W;
        float v = ((float)y + 0.5f - cy) * 2.f * tanfovy / (float)H;
        for (int k = 0; k < 3; ++k) {
            rd[k * P + q] = c2w[4 * k] * u + c2w[4 * k + 1] * v + c2w[4 * k + 2];
            pts[k * P + q] = c2w[4 * k + 3] + rd[k * P + q] * depth[q];
        }
    }
    const float inv_hw = 1.f / (float)P;
    double loss = 0.0;
    for (int y = pad; y < H - pad; ++y) for (int x = pad; x < W - pad; ++x) {
        int64_t q = (int64_t)y * W + x;
        int64_t xp = q + pad, xm = q - pad, yp = q + (int64_t)pad * W, ym = q - (int64_t)pad * W;
        float dx[3], dy[3], c[3], n[3];
        for (int k = 0; k < 3; ++k) { dx[k] = pts[k * P + xp] - pts[k * P + xm]; dy[k] = pts[k * P + yp] - pts[k * P + ym]; }
        c[0] = dx[1] * dy[2] - dx[2] * dy[1];
        c[1] = dx[2] * dy[0] - dx[0] * dy[2];
        c[2] = dx[0] * dy[1] - dx[1] * dy[0];
        float cn = sqrtf(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
        float den = cn > 1e-12f ? cn : 1e-12f;
        for (int k = 0; k < 3; ++k) n[k] = c[k] / den;
        float s = 1.f;
        if (tol_cos > 0.f) {
            float pd[3];
            for (int k = 0; k < 3; ++k) pd[k] = pts[k * P + q] - c2w[4 * k + 3];
            float pn = sqrtf(pd[0] * pd[0] + pd[1] * pd[1] + pd[2] * pd[2]);
            pn = pn > 1e-12f ? pn : 1e-12f;
            float dot = n[0] * (pd[0] / pn) + n[1] * (pd[1] / pn) + n[2] * (pd[2] / pn);
            if (!(dot > tol_cos)) s = 0.f;
        }
        float alpha = T ? 1.f - T[q] : 1.f;
        if (T) s *= alpha;
        float N[3] = {-n[0] * s, -n[1] * s, -n[2] * s};
        if (!(N[0] != 0.f || N[1] != 0.f || N[2] != 0.f)) continue;
        float target = T ? alpha * alpha : 1.f;
        float dotn = nr[q] * N[0] + nr[P + q] * N[1] + nr[2 * P + q] * N[2];
        loss += (double)(target - dotn);
        for (int k = 0; k < 3; ++k) grad_normal[k * P + q] += -N[k] * inv_hw;
        /* dL/dn = s * n_r / HW; through the clamped normalisation; then dc = dx x dy */
        float g[3], gc[3];
        for (int k = 0; k < 3; ++k) g[k] = s * nr[k * P + q] * inv_hw;
        if (cn > 1e-12f) {
            float ng = n[0] * g[0] + n[1] * g[1] + n[2] * g[2];
            for (int k = 0; k < 3; ++k) gc[k] = (g[k] - n[k] * ng) / cn;
        } else {
            for (int k = 0; k < 3; ++k) gc[k] = g[k] / 1e-12f;
        }
        float* a = gdx + q; float* b = gdy + q;
        a[0] += dy[1] * gc[2] - dy[2] * gc[1];          /* dL/ddx = dy x gc */
        a[P] += dy[2] * gc[0] - dy[0] * gc[2];
        a[2 * P] += dy[0] * gc[1] - dy[1] * gc[0];
        b[0] += gc[1] * dx[2] - gc[2] * dx[1];          /* dL/ddy = gc x dx */
        b[P] += gc[2] * dx[0] - gc[0] * dx[2];
        b[2 * P] += gc[0] * dx[1] - gc[1] * dx[0];
    }
    for (int y = 0; y < H; ++y) for (int x = 0; x < W; ++x) {
        int64_t q = (int64_t)y * W + x;
        float gp[3] = {0.f, 0.f, 0.f};
        for (int k = 0; k < 3; ++k) {
            if (x - pad >= 0) gp[k] += gdx[k * P + q - pad];
            if (x + pad < W) gp[k] -= gdx[k * P + q + pad];
            if (y - pad >= 0) gp[k] += gdy[k * P + q - (int64_t)pad * W];
            if (y + pad < H) gp[k] -= gdy[k * P + q + (int64_t)pad * W];
        }
        grad_depth[q] += rd[q] * gp[0] + rd[P + q] * gp[1] + rd[2 * P + q] * gp[2];
    }
    free(rd); free(pts); free(gdx); free(gdy);
    return loss / (double)P;
}

/* ------------------------------------------------------------------ Adam
 * cuda/src/adam_step.cu:21-159 (host bias corrections in double). */
static inline float lerp_(float v0, float v1, float t) { return fmaf(t, v1, fmaf(-t, v0, v0)); }

void svo_adam(int n, int biased, int sparse, float* p, const float* g, float* m, float* v, double step,
              double lr, double beta1, double beta2, float eps) {
    float step_size, rbc2;
    if (biased) { step_size = (float)lr; rbc2 = 1.f; }
    else {
        double bc1 = 1.0 - pow(beta1, step), bc2 = 1.0 - pow(beta2, step);
        step_size = (float)(lr / bc1); rbc2 = (float)(1.0 / sqrt(bc2));
    }
    float b1 = (float)beta1, b2 = (float)beta2;
    for (int i = 0; i < n; ++i) {
        float gv = g[i];
        if (sparse && gv == 0.0f) continue;
        float mv = lerp_(gv, m[i], b1), vv = lerp_(gv * gv, v[i], b2);
        float den = biased ? sqrtf(vv) + eps : fmaf(sqrtf(vv), rbc2, eps);
        p[i] -= step_size * (mv / den);
        m[i] = mv; v[i] = vv;
    }
}
