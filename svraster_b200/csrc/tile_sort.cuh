// Binning of the sorted (tile, voxel, octant) records without a global radix sort.
//
// The reference emits one (key, value) per (octant, tile) of every rendered voxel, key =
// tile << 48 | rank with rank = octree path ^ repeat3(octant), and sorts all records with a
// stable 64-bit radix sort (cuda/src/forward.cu:749-802, 882-939): within a tile, records
// are ordered by rank and then by emission order (voxel id, then octant).  Here:
//
//  * once per octree, every (voxel, octant) pair gets its position in that order among all
//    8N pairs (the pair-order table: full 48-bit rank, ties by voxel id then octant);
//  * per step, records are counted per tile (one shared-memory histogram per view and CTA,
//    one global atomic per touched tile), the counts are scanned into tile ranges (which
//    also yields the heavy-first tile launch order), and every record is scattered into its
//    tile's range at a position taken by atomics, so unordered;
//  * one CTA per tile then sorts its records by their pair position, a key unique within
//    the tile, so the result is exactly the reference's order whatever order the scatter
//    left: 8-bit LSD passes, each a stable warp multisplit (digit peers from eight ballots)
//    and a block scan, in registers and shared memory for a tile of at most TS_CHUNK
//    records.  A larger tile is first split, unordered, into 256 buckets on its top 8 key
//    bits (keys are unique, so no stability is needed there); runs of consecutive buckets of
//    at most TS_CHUNK records are then sorted in shared memory over the bits below the split
//    digit, a bigger bucket is split again, and past two splits sorted by LSD passes over
//    global memory.
//  * the pair-order table is octant-major (entry q*N + voxel), so the scatter reads it
//    coalesced.
#pragma once

#include "svr_common.cuh"

namespace svr {

constexpr int TS_THREADS = 256;               // threads of the per-tile sort (one per digit)
constexpr int TS_WARPS = TS_THREADS / 32;
constexpr int TS_K = 16;                      // keys per thread of one block-tile
constexpr int TS_CHUNK = TS_THREADS * TS_K;   // records sorted in shared memory (4096)
constexpr int TS_BLK = 2048;                  // tiles per CTA of the tile scan
constexpr unsigned FULL = 0xffffffffu;

struct TileSortSmem {
    uint32_t whist[TS_WARPS][256];   // per-warp digit counts, then per-warp digit bases
    uint32_t base[256];              // running digit base (global path), bucket cursors (split)
    uint32_t wsum[TS_WARPS];
    uint32_t b_off[2][256];          // bucket offsets of the two split levels
    uint32_t b_cnt[2][256];          // bucket sizes of the two split levels
    uint32_t key[TS_CHUNK];          // shared-memory path: keys of the tile between passes
    uint32_t val[TS_CHUNK];
};

// Lanes of the warp holding the same 8-bit digit as this lane (this lane included when
// valid): the AND over the digit's bits of the matching ballot or its complement.
__device__ __forceinline__ uint32_t digit_peers(uint32_t d, bool valid) {
    uint32_t peers = __ballot_sync(FULL, valid);
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        const uint32_t bal = __ballot_sync(FULL, (d >> b) & 1u);
        peers &= ((d >> b) & 1u) ? bal : ~bal;
    }
    return peers;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Exclusive scan of one value per thread over the 256 threads of the CTA; returns the
// thread's exclusive prefix, `total` gets the sum.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* wsum, uint32_t& total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    uint32_t wbase = 0, tot = 0;
#pragma unroll
    for (int i = 0; i < TS_WARPS; ++i) {
        const uint32_t s = wsum[i];
        if (i < w) wbase += s;
        tot += s;
    }
    __syncthreads();
    total = tot;
    return wbase + x - v;
}

// Stable rank of one block-tile (K keys per thread at warp-striped positions w*32*K + k*32 +
// lane, the first `count` valid) by digit (key >> sh) & 255.  On return pos[k] is the key's
// destination: base[d] + its rank among the block-tile's digit-d keys, where base is the
// exclusive scan of the block-tile's own digit counts (self_scan) or the running base in
// S.base, which is then advanced past this block-tile.
template <int K>
__device__ __forceinline__ void block_rank(const uint32_t (&key)[K], int count, int sh, bool self_scan,
                                           TileSortSmem& S, uint32_t (&pos)[K]) {
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    for (int i = tid; i < TS_WARPS * 256; i += TS_THREADS) (&S.whist[0][0])[i] = 0u;
    __syncthreads();
    uint32_t* wh = S.whist[w];
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int i = w * 32 * K + k * 32 + lane;
        const bool valid = i < count;
        const uint32_t d = (key[k] >> sh) & 255u;
        const uint32_t peers = digit_peers(d, valid);
        uint32_t before = 0u;
        if (valid) before = wh[d];
        pos[k] = before + __popc(peers & lt);
        __syncwarp();
        if (valid && lane == 31 - __clz(peers)) wh[d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // thread t owns digit t: per-warp bases in warp order
    uint32_t tot = 0;
#pragma unroll
    for (int ww = 0; ww < TS_WARPS; ++ww) tot += S.whist[ww][tid];
    uint32_t run;
    if (self_scan) {
        uint32_t all;
        run = block_exclusive_scan(tot, S.wsum, all);
    } else {
        run = S.base[tid];
        S.base[tid] = run + tot;
    }
#pragma unroll
    for (int ww = 0; ww < TS_WARPS; ++ww) {
        const uint32_t v = S.whist[ww][tid];
        S.whist[ww][tid] = run;
        run += v;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int i = w * 32 * K + k * 32 + lane;
        if (i < count) pos[k] += wh[(key[k] >> sh) & 255u];
    }
}

// n <= K * TS_THREADS records of A[start, start + n) sorted in registers (K keys per thread) by
// key - kbase over npass 8-bit digits, with shared memory between the LSD passes; writes the
// sorted values and the tile id of every record at the same positions.
template <int K>
__device__ __forceinline__ void sort_in_smem(const uint2* __restrict__ A, uint32_t start, int n, int npass,
                                             uint32_t kbase, int tile, TileSortSmem& S,
                                             uint32_t* __restrict__ vals_out, uint32_t* __restrict__ tile_out,
                                             unsigned* __restrict__ status)
{
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    uint32_t key[K], val[K], pos[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int i = w * 32 * K + k * 32 + lane;
        const uint2 kv = i < n ? A[start + i] : make_uint2(kbase, 0u);
        key[k] = kv.x - kbase;
        val[k] = kv.y;
    }
    for (int p = 0; p < npass; ++p) {
        block_rank<K>(key, n, 8 * p, true, S, pos);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int i = w * 32 * K + k * 32 + lane;
            if (i < n) {
                if (pos[k] < (uint32_t)n) { S.key[pos[k]] = key[k]; S.val[pos[k]] = val[k]; }
                else atomicOr(status, ERR_COUNT_MISMATCH);
            }
        }
        __syncthreads();
        if (p == npass - 1) break;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int i = w * 32 * K + k * 32 + lane;
            key[k] = i < n ? S.key[i] : 0u;
            val[k] = i < n ? S.val[i] : 0u;
        }
        __syncthreads();
    }
    for (int i = tid; i < n; i += TS_THREADS) {
        vals_out[start + i] = S.val[i];
        tile_out[start + i] = (uint32_t)tile;
    }
}

// The smallest K-per-thread instance of sort_in_smem that holds n <= TS_CHUNK records.
__device__ __forceinline__ void sort_chunk(const uint2* __restrict__ A, uint32_t start, int n, int npass,
                                           uint32_t kbase, int tile, TileSortSmem& S,
                                           uint32_t* __restrict__ vals_out, uint32_t* __restrict__ tile_out,
                                           unsigned* __restrict__ status)
{
    if (n <= TS_THREADS) sort_in_smem<1>(A, start, n, npass, kbase, tile, S, vals_out, tile_out, status);
    else if (n <= 2 * TS_THREADS) sort_in_smem<2>(A, start, n, npass, kbase, tile, S, vals_out, tile_out, status);
    else if (n <= 4 * TS_THREADS) sort_in_smem<4>(A, start, n, npass, kbase, tile, S, vals_out, tile_out, status);
    else if (n <= 8 * TS_THREADS) sort_in_smem<8>(A, start, n, npass, kbase, tile, S, vals_out, tile_out, status);
    else sort_in_smem<TS_K>(A, start, n, npass, kbase, tile, S, vals_out, tile_out, status);
}

// Unordered split of src[start, start + n) by the digit (key >> sh) & 255 into
// dst[start, start + n), bucket after bucket: the bucket sizes and offsets (from start) go to
// S.b_cnt[lv] / S.b_off[lv].  Keys are unique within a tile, so the order inside a bucket is
// left to the bucket's own sort.  A warp's lanes of one digit take one shared-memory atomic.
constexpr int SPLIT_K = 8;   // keys per thread per round of the split
__device__ __forceinline__ void msd_split(const uint2* __restrict__ src, uint2* __restrict__ dst, uint32_t start,
                                          int n, int sh, int lv, TileSortSmem& S, unsigned* __restrict__ status)
{
    const int tid = threadIdx.x, lane = tid & 31;
    const uint32_t lt = lanemask_lt();
    S.base[tid] = 0u;
    __syncthreads();
    for (int c0 = 0; c0 < n; c0 += TS_THREADS * SPLIT_K) {
        uint32_t d[SPLIT_K];
#pragma unroll
        for (int k = 0; k < SPLIT_K; ++k) {
            const int i = c0 + k * TS_THREADS + tid;
            d[k] = i < n ? (src[start + i].x >> sh) & 255u : 0u;
        }
#pragma unroll
        for (int k = 0; k < SPLIT_K; ++k) {
            const bool valid = c0 + k * TS_THREADS + tid < n;
            const uint32_t peers = digit_peers(d[k], valid);
            if (valid && lane == 31 - __clz(peers)) atomicAdd(&S.base[d[k]], (uint32_t)__popc(peers));
        }
    }
    __syncthreads();
    {
        const uint32_t c = S.base[tid];
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan(c, S.wsum, tot);
        S.b_cnt[lv][tid] = c;
        S.b_off[lv][tid] = ex;
        S.base[tid] = ex;
    }
    __syncthreads();
    for (int c0 = 0; c0 < n; c0 += TS_THREADS * SPLIT_K) {
        uint2 kv[SPLIT_K];
#pragma unroll
        for (int k = 0; k < SPLIT_K; ++k) {
            const int i = c0 + k * TS_THREADS + tid;
            kv[k] = i < n ? src[start + i] : make_uint2(0u, 0u);
        }
#pragma unroll
        for (int k = 0; k < SPLIT_K; ++k) {
            const bool valid = c0 + k * TS_THREADS + tid < n;
            const uint32_t d = (kv[k].x >> sh) & 255u;
            const uint32_t peers = digit_peers(d, valid);
            const int leader = 31 - __clz(peers);
            uint32_t b = 0u;
            if (valid && lane == leader) b = atomicAdd(&S.base[d], (uint32_t)__popc(peers));
            b = __shfl_sync(FULL, b, leader & 31);
            if (valid) {
                const uint32_t pos = b + __popc(peers & lt);
                if (pos < (uint32_t)n) dst[start + pos] = kv[k];
                else atomicOr(status, ERR_COUNT_MISMATCH);
            }
        }
    }
    __syncthreads();
}

// LSD sort of src[start, start + n) (any size) over npass 8-bit digits in passes over global
// memory, ping-pong with dst; the last pass writes the values and tile ids.  Each pass counts
// the digits over the whole range, then ranks and scatters it block-tile by block-tile with a
// running digit base.
__device__ __forceinline__ void lsd_global(uint2* __restrict__ src, uint2* __restrict__ dst, uint32_t start, int n,
                                           int npass, int tile, TileSortSmem& S, uint32_t* __restrict__ vals_out,
                                           uint32_t* __restrict__ tile_out, unsigned* __restrict__ status)
{
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    uint32_t key[TS_K], val[TS_K], pos[TS_K];
    for (int p = 0; p < npass; ++p) {
        const int sh = 8 * p;
        const bool last = p == npass - 1;
        S.base[tid] = 0u;
        __syncthreads();
        for (int c0 = 0; c0 < n; c0 += TS_CHUNK) {
            const int cnt = min(TS_CHUNK, n - c0);
#pragma unroll
            for (int k = 0; k < TS_K; ++k) {
                const int i = w * 32 * TS_K + k * 32 + lane;
                const bool valid = i < cnt;
                const uint32_t d = valid ? (src[start + c0 + i].x >> sh) & 255u : 0u;
                const uint32_t peers = digit_peers(d, valid);
                if (valid && lane == 31 - __clz(peers)) atomicAdd(&S.base[d], (uint32_t)__popc(peers));
            }
        }
        __syncthreads();
        {
            uint32_t all;
            const uint32_t ex = block_exclusive_scan(S.base[tid], S.wsum, all);
            __syncthreads();
            S.base[tid] = ex;
            __syncthreads();
        }
        for (int c0 = 0; c0 < n; c0 += TS_CHUNK) {
            const int cnt = min(TS_CHUNK, n - c0);
#pragma unroll
            for (int k = 0; k < TS_K; ++k) {
                const int i = w * 32 * TS_K + k * 32 + lane;
                const uint2 kv = i < cnt ? src[start + c0 + i] : make_uint2(0u, 0u);
                key[k] = kv.x;
                val[k] = kv.y;
            }
            block_rank(key, cnt, sh, false, S, pos);
#pragma unroll
            for (int k = 0; k < TS_K; ++k) {
                const int i = w * 32 * TS_K + k * 32 + lane;
                if (i < cnt && pos[k] >= (uint32_t)n) atomicOr(status, ERR_COUNT_MISMATCH);
                else if (i < cnt) {
                    if (last) {
                        vals_out[start + pos[k]] = val[k];
                        tile_out[start + pos[k]] = (uint32_t)tile;
                    } else {
                        dst[start + pos[k]] = make_uint2(key[k], val[k]);
                    }
                }
            }
            __syncthreads();
        }
        uint2* t = src; src = dst; dst = t;
    }
}

// The buckets of split level LV of src[start, ...): runs of consecutive buckets of at most
// TS_CHUNK records in all are sorted in shared memory by key - (their first key's digits), over
// the bits below the split digit plus those of the run's digit span; a bucket above TS_CHUNK is
// split again on the next 8 bits (level 1) or, past two levels, sorted by global passes.  Every
// thread walks the same buckets (shared-memory sizes), so the barriers inside are uniform.
template <int LV>
__device__ void sort_buckets(uint2* __restrict__ src, uint2* __restrict__ alt, uint32_t start, int sh,
                             uint32_t prefix, int tile, TileSortSmem& S, uint32_t* __restrict__ vals_out,
                             uint32_t* __restrict__ tile_out, unsigned* __restrict__ status)
{
    int b = 0;
    while (b < 256) {
        const uint32_t c = S.b_cnt[LV][b];
        if (c == 0u) { ++b; continue; }
        const uint32_t o = start + S.b_off[LV][b];
        if (c > (uint32_t)TS_CHUNK) {
            if constexpr (LV == 0) {
                if (sh > 0) {
                    const int sh2 = sh > 8 ? sh - 8 : 0;
                    msd_split(src, alt, o, (int)c, sh2, 1, S, status);
                    sort_buckets<1>(alt, src, o, sh2, prefix | ((uint32_t)b << sh), tile, S, vals_out, tile_out,
                                    status);
                    ++b;
                    continue;
                }
            }
            lsd_global(src, alt, o, (int)c, max(1, (sh + 7) / 8), tile, S, vals_out, tile_out, status);
            ++b;
            continue;
        }
        int e = b + 1, last = b;
        uint32_t sum = c;
        while (e < 256) {
            const uint32_t ce = S.b_cnt[LV][e];
            if (ce > (uint32_t)TS_CHUNK || sum + ce > (uint32_t)TS_CHUNK) break;
            if (ce) { sum += ce; last = e; }
            ++e;
        }
        // keys of the run: prefix | digit << sh | low bits, digit in [b, last]
        const uint64_t span = ((uint64_t)(last - b + 1) << sh) - 1u;
        const int bits = span ? 64 - __clzll((long long)span) : 0;
        sort_chunk(src, o, (int)sum, max(1, (bits + 7) / 8), prefix | ((uint32_t)b << sh), tile, S, vals_out,
                   tile_out, status);
        b = e;
    }
}

// Sort of one tile's records [start, start + n) by key (pair position), values along.
// Input in A as (key, value) pairs; the sorted values go to vals_out and the tile id of every
// record to tile_out.  A tile of at most TS_CHUNK records is sorted in shared memory; a larger
// one is split on its top 8 key bits into B, bucket runs are then sorted in shared memory
// (sort_buckets), with A as scratch.
#ifndef SVR_TS_MINB
#define SVR_TS_MINB 2
#endif
__global__ void __launch_bounds__(TS_THREADS, SVR_TS_MINB) tile_sort_kernel(
    int T, const uint32_t* __restrict__ order, const uint2* __restrict__ ranges, int key_bits,
    uint2* __restrict__ A, uint2* __restrict__ B,
    uint32_t* __restrict__ vals_out, uint32_t* __restrict__ tile_out, unsigned* __restrict__ status)
{
    extern __shared__ __align__(16) unsigned char ts_smem[];
    TileSortSmem& S = *reinterpret_cast<TileSortSmem*>(ts_smem);
    const int tile = order ? (int)order[blockIdx.x] : (int)blockIdx.x;
    if (tile >= T) return;
    const uint2 rg = ranges[tile];
    if (rg.y <= rg.x) return;
    const uint32_t start = rg.x;
    const int n = (int)(rg.y - rg.x);
    if (n <= TS_CHUNK) {
        sort_chunk(A, start, n, max(1, (key_bits + 7) / 8), 0u, tile, S, vals_out, tile_out, status);
        return;
    }
    const int sh = key_bits > 8 ? key_bits - 8 : 0;
    msd_split(A, B, start, n, sh, 0, S, status);
    sort_buckets<0>(B, A, start, sh, 0u, tile, S, vals_out, tile_out, status);
}
}  // namespace svr

namespace svr {

// Tile rectangle of a rendered item (auxiliary.h:97-111, as in preprocess).
__device__ __forceinline__ void item_rect(const uint2 bb, int gx, int gy, int& tx0, int& ty0, int& tx1, int& ty1) {
    tx0 = max(0, min(gx - 1, (int)((bb.x >> 16) / TILE)));
    ty0 = max(0, min(gy - 1, (int)((bb.x << 16 >> 16) / TILE)));
    tx1 = max(0, min(gx - 1, (int)((bb.y >> 16) / TILE)));
    ty1 = max(0, min(gy - 1, (int)((bb.y << 16 >> 16) / TILE)));
}

// Items per thread per round of the count and scatter loops: their loads are issued together.
constexpr int ITEM_U = 4;

// The rendered items among v0 + tid + u * blockDim.x (u < ITEM_U, below v1) of view vi: octant
// bits (0 = not rendered) and bbox.
__device__ __forceinline__ void load_items(int i0, int v1, int vi, int N, const uint32_t* __restrict__ ndup,
                                           const uint2* __restrict__ bboxes, const uint32_t* __restrict__ bits,
                                           uint32_t (&qb)[ITEM_U], uint2 (&bb)[ITEM_U])
{
    uint32_t nd[ITEM_U];
#pragma unroll
    for (int u = 0; u < ITEM_U; ++u) {
        const int i = i0 + u * (int)blockDim.x;
        nd[u] = i < v1 ? ndup[(size_t)vi * N + i] : 0u;
    }
#pragma unroll
    for (int u = 0; u < ITEM_U; ++u) {
        const size_t item = (size_t)vi * N + i0 + u * (int)blockDim.x;
        qb[u] = nd[u] ? bits[item] : 0u;
        bb[u] = nd[u] ? bboxes[item] : make_uint2(0u, 0u);
    }
}

// Records per tile.  Grid (chunks, views): each CTA visits a range of the voxels of view
// blockIdx.y, adds the octant count of every rendered item to each tile of its rectangle in
// a shared-memory histogram of the view's tiles (SMEM; else straight to global memory), and
// flushes the non-zero entries with one global atomic each; with `chist` it also stores the
// whole histogram (row blockIdx.x of a [gridDim.x, T] array), which the scatter then reads
// instead of counting its records again.
template <bool SMEM>
__global__ void __launch_bounds__(256) tile_count_kernel(
    const __grid_constant__ Views V, int N, const uint32_t* __restrict__ ndup, const uint2* __restrict__ bboxes,
    const uint32_t* __restrict__ bits, uint32_t* __restrict__ tile_cnt, uint32_t* __restrict__ chist, int T)
{
    extern __shared__ __align__(16) uint32_t hist[];
    const int vi = blockIdx.y;
    const svr_view_t& view = V.v[vi];
    const int gx = view.tiles_x, gy = view.tiles_y, nt = gx * gy;
    uint32_t* cnt = SMEM ? hist : tile_cnt + view.tile_offset;
    if (SMEM) {
        for (int i = threadIdx.x; i < nt; i += blockDim.x) hist[i] = 0u;
        __syncthreads();
    }
    const int per = (N + gridDim.x - 1) / gridDim.x;
    const int v0 = blockIdx.x * per, v1 = min(N, v0 + per);
    for (int i0 = v0 + threadIdx.x; i0 < v1; i0 += ITEM_U * blockDim.x) {
        uint32_t qb[ITEM_U];
        uint2 bb[ITEM_U];
        load_items(i0, v1, vi, N, ndup, bboxes, bits, qb, bb);
#pragma unroll
        for (int u = 0; u < ITEM_U; ++u) {
            if (!qb[u]) continue;
            const uint32_t k = __popc(qb[u]);
            int tx0, ty0, tx1, ty1;
            item_rect(bb[u], gx, gy, tx0, ty0, tx1, ty1);
            for (int y = ty0; y <= ty1; ++y)
                for (int x = tx0; x <= tx1; ++x) atomicAdd(&cnt[y * gx + x], k);
        }
    }
    if (SMEM) {
        __syncthreads();
        // chist (when given): the CTA's whole histogram, row blockIdx.x, for the scatter
        uint32_t* row = chist ? chist + (size_t)blockIdx.x * T + view.tile_offset : nullptr;
        for (int i = threadIdx.x; i < nt; i += blockDim.x) {
            const uint32_t c = hist[i];
            if (c) atomicAdd(&tile_cnt[view.tile_offset + i], c);
            if (row) row[i] = c;
        }
    }
}

// Heavy-first launch bucket of a tile: 8 steps per octave of its record count, most first;
// empty tiles last.
__device__ __forceinline__ uint32_t heavy_bucket(uint32_t c) {
    if (c == 0u) return 255u;
    const uint32_t e = 31u - __clz(c);
    const uint32_t m = e >= 3u ? (c >> (e - 3u)) & 7u : (c << (3u - e)) & 7u;
    const uint32_t code = min(e * 8u + m, 254u);
    return 254u - code;
}

// Scan of the tile counts, first half: per CTA of TS_BLK tiles the record sum and the
// histogram of launch buckets.
__global__ void __launch_bounds__(256) tile_sum_kernel(int T, const uint32_t* __restrict__ tile_cnt,
                                                      uint32_t* __restrict__ blk_sum, uint32_t* __restrict__ blk_hist)
{
    __shared__ uint32_t h[256];
    __shared__ uint32_t ws[8];
    h[threadIdx.x] = 0u;
    __syncthreads();
    uint32_t s = 0;
    for (int j = 0; j < TS_BLK / 256; ++j) {
        const int t = blockIdx.x * TS_BLK + j * 256 + threadIdx.x;
        const uint32_t c = t < T ? tile_cnt[t] : 0u;
        s += c;
        if (t < T) atomicAdd(&h[heavy_bucket(c)], 1u);
    }
    s = __reduce_add_sync(FULL, s);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t tot = 0;
        for (int i = 0; i < 8; ++i) tot += ws[i];
        blk_sum[blockIdx.x] = tot;
    }
    blk_hist[(size_t)blockIdx.x * 256 + threadIdx.x] = h[threadIdx.x];
}

// Scan of the tile counts, second half: tile ranges clipped to the capacity, the scatter
// cursors (range starts), the record count of the batch, and the heavy-first launch order
// (stable by tile index within a bucket).
__global__ void __launch_bounds__(256) tile_offsets_kernel(
    int T, int nblk, const uint32_t* __restrict__ tile_cnt, const uint32_t* __restrict__ blk_sum,
    const uint32_t* __restrict__ blk_hist, int64_t cap, uint2* __restrict__ ranges, uint32_t* __restrict__ cursor,
    uint32_t* __restrict__ order, long long* __restrict__ count_out, int* __restrict__ meta_bits,
    unsigned* __restrict__ status)
{
    __shared__ uint32_t wsum[TS_WARPS];
    __shared__ uint32_t bbase[256];
    __shared__ uint32_t whist[TS_WARPS][256];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    // records before this CTA's tiles, and the batch total
    unsigned long long before = 0, total = 0;
    for (int b = 0; b < nblk; ++b) {
        const uint32_t s = blk_sum[b];
        if (b < (int)blockIdx.x) before += s;
        total += s;
    }
    // launch-bucket base of this CTA: tiles of heavier buckets, then this bucket's tiles in
    // earlier CTAs
    {
        uint32_t mine = 0, all = 0;
        for (int b = 0; b < nblk; ++b) {
            const uint32_t h = blk_hist[(size_t)b * 256 + tid];
            if (b < (int)blockIdx.x) mine += h;
            all += h;
        }
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan(all, wsum, tot);
        bbase[tid] = ex + mine;
    }
    for (int i = tid; i < TS_WARPS * 256; i += 256) (&whist[0][0])[i] = 0u;
    __syncthreads();
    // this CTA's TS_BLK tiles, 8 per thread, warp-striped: tile t0 + w*256 + k*32 + lane
    constexpr int KT = TS_BLK / 256;
    const int t0 = blockIdx.x * TS_BLK;
    uint32_t c[KT], rk[KT];
    uint32_t run = 0;
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < KT; ++k) {
        const int t = t0 + w * 32 * KT + k * 32 + lane;
        c[k] = t < T ? tile_cnt[t] : 0u;
        // running exclusive prefix of the counts inside the warp
        uint32_t x = c[k];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(FULL, x, o);
            if (lane >= o) x += y;
        }
        rk[k] = run + x - c[k];
        run += __shfl_sync(FULL, x, 31);
    }
    // warp totals -> warp bases
    uint32_t tot;
    const uint32_t wex = block_exclusive_scan(lane == 0 ? run : 0u, wsum, tot);
    const uint32_t wbase = __shfl_sync(FULL, wex, 0);
#pragma unroll
    for (int k = 0; k < KT; ++k) {
        const int t = t0 + w * 32 * KT + k * 32 + lane;
        if (t >= T) continue;
        const unsigned long long s0 = before + wbase + rk[k];
        const unsigned long long s1 = s0 + c[k];
        const uint32_t a = (uint32_t)min(s0, (unsigned long long)cap);
        const uint32_t e = (uint32_t)min(s1, (unsigned long long)cap);
        ranges[t] = e > a ? make_uint2(a, e) : make_uint2(0u, 0u);   // empty tiles: [0, 0), as the reference
        cursor[t] = (uint32_t)min(s0, (unsigned long long)0xFFFFFFFFull);
    }
    // stable rank of the tiles by launch bucket (warp multisplit, then across warps)
    uint32_t d[KT], pos[KT];
#pragma unroll
    for (int k = 0; k < KT; ++k) {
        const int t = t0 + w * 32 * KT + k * 32 + lane;
        const bool valid = t < T;
        d[k] = heavy_bucket(c[k]);
        const uint32_t peers = digit_peers(d[k], valid);
        uint32_t b4 = 0u;
        if (valid) b4 = whist[w][d[k]];
        pos[k] = b4 + __popc(peers & lt);
        __syncwarp();
        if (valid && lane == 31 - __clz(peers)) whist[w][d[k]] = b4 + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    {
        uint32_t r = bbase[tid];
        for (int ww = 0; ww < TS_WARPS; ++ww) {
            const uint32_t v = whist[ww][tid];
            whist[ww][tid] = r;
            r += v;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < KT; ++k) {
        const int t = t0 + w * 32 * KT + k * 32 + lane;
        if (t < T) {
            const uint32_t o = whist[w][d[k]] + pos[k];
            if (o < (uint32_t)T) order[o] = (uint32_t)t;
            else atomicOr(status, ERR_COUNT_MISMATCH);
        }
    }
    if (blockIdx.x == 0 && tid == 0) {
        *count_out = total < (unsigned long long)cap ? (long long)total : (long long)cap;
        meta_bits[0] = 0;   // the sorted "keys" are plain tile ids
        meta_bits[1] = 0;
        if (total > (unsigned long long)cap) atomicOr(status, ERR_CAPACITY);
        if (total >= (1ull << 32)) atomicOr(status, ERR_CAPACITY);
    }
}

// Scatter of the records into their tiles' ranges.  Same grid and histogram as
// tile_count_kernel: the CTA takes its records per tile from the count kernel's stored
// histogram (chist) or counts them again, reserves one contiguous run per
// touched tile with a global atomic on the tile's cursor, then places every record inside
// its run with a shared-memory atomic.  Key = the (voxel, octant) pair's position in the
// reference order (pair-order table), value = octant << 29 | voxel id, stored together.
template <bool SMEM>
__global__ void __launch_bounds__(256) tile_scatter_kernel(
    const __grid_constant__ Views V, int N, const uint32_t* __restrict__ ndup, const uint2* __restrict__ bboxes,
    const uint32_t* __restrict__ bits, const uint32_t* __restrict__ pair_pos, uint32_t* __restrict__ cursor,
    int64_t cap, uint2* __restrict__ kv, const uint32_t* __restrict__ chist, int T, unsigned* __restrict__ status)
{
    extern __shared__ __align__(16) uint32_t hist[];
    const int vi = blockIdx.y;
    const svr_view_t& view = V.v[vi];
    const int gx = view.tiles_x, gy = view.tiles_y, nt = gx * gy;
    const int per = (N + gridDim.x - 1) / gridDim.x;
    const int v0 = blockIdx.x * per, v1 = min(N, v0 + per);
    if (SMEM) {
        if (chist) {
            // the count kernel's histogram of this CTA's records (same grid, same voxel range)
            const uint32_t* row = chist + (size_t)blockIdx.x * T + view.tile_offset;
            for (int i = threadIdx.x; i < nt; i += blockDim.x) hist[i] = row[i];
        } else {
            for (int i = threadIdx.x; i < nt; i += blockDim.x) hist[i] = 0u;
            __syncthreads();
            for (int i0 = v0 + threadIdx.x; i0 < v1; i0 += ITEM_U * blockDim.x) {
                uint32_t qb[ITEM_U];
                uint2 bb[ITEM_U];
                load_items(i0, v1, vi, N, ndup, bboxes, bits, qb, bb);
#pragma unroll
                for (int u = 0; u < ITEM_U; ++u) {
                    if (!qb[u]) continue;
                    const uint32_t k = __popc(qb[u]);
                    int tx0, ty0, tx1, ty1;
                    item_rect(bb[u], gx, gy, tx0, ty0, tx1, ty1);
                    for (int y = ty0; y <= ty1; ++y)
                        for (int x = tx0; x <= tx1; ++x) atomicAdd(&hist[y * gx + x], k);
                }
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < nt; i += blockDim.x) {
            const uint32_t h = hist[i];
            if (h) hist[i] = atomicAdd(&cursor[view.tile_offset + i], h);
        }
        __syncthreads();
    }
    for (int i0 = v0 + threadIdx.x; i0 < v1; i0 += ITEM_U * blockDim.x) {
        uint32_t qb[ITEM_U];
        uint2 bb[ITEM_U];
        load_items(i0, v1, vi, N, ndup, bboxes, bits, qb, bb);
        // pair positions of the first octant of every item (most items have one)
        uint32_t p0[ITEM_U];
#pragma unroll
        for (int u = 0; u < ITEM_U; ++u)
            p0[u] = qb[u] ? pair_pos[(size_t)(__ffs(qb[u]) - 1) * N + i0 + u * (int)blockDim.x] : 0u;
#pragma unroll
        for (int u = 0; u < ITEM_U; ++u) {
            if (!qb[u]) continue;
            const int i = i0 + u * (int)blockDim.x;
            const uint32_t q_first = (uint32_t)__ffs(qb[u]) - 1u;
            const uint32_t k = __popc(qb[u]);
            uint32_t pp[8];
#pragma unroll
            for (int q = 0; q < 8; ++q)
                pp[q] = (uint32_t)q == q_first ? p0[u] : ((qb[u] >> q) & 1u ? pair_pos[(size_t)q * N + i] : 0u);
            int tx0, ty0, tx1, ty1;
            item_rect(bb[u], gx, gy, tx0, ty0, tx1, ty1);
            for (int y = ty0; y <= ty1; ++y)
                for (int x = tx0; x <= tx1; ++x) {
                    const int lt_ = y * gx + x;
                    uint32_t p = SMEM ? atomicAdd(&hist[lt_], k) : atomicAdd(&cursor[view.tile_offset + lt_], k);
#pragma unroll
                    for (uint32_t q = 0; q < 8; ++q) {
                        if (!(qb[u] & (1u << q))) continue;
                        if ((int64_t)p < cap) kv[p] = make_uint2(pp[q], (q << 29) | (uint32_t)i);
                        ++p;
                    }
                }
        }
    }
}

// Pair-order table (once per octree): position of every (voxel, octant) pair in the order of
// the full 48-bit rank, ties by voxel id then octant (the reference's stable order).
__global__ void pair_rank_kernel(int64_t N, const int64_t* __restrict__ octpaths, uint64_t* __restrict__ keys,
                                 uint32_t* __restrict__ vals)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= 8 * N) return;
    const uint64_t q = (uint64_t)(s & 7);
    uint64_t rep = 0;
#pragma unroll
    for (int l = 0; l < MAX_LEVELS; ++l) rep = (rep << 3) | q;
    keys[s] = (uint64_t)octpaths[s >> 3] ^ rep;
    vals[s] = (uint32_t)s;
}

// Octant-major table: entry q*N + v, so the items of a view (mostly one octant over a run of
// voxel ids) read it coalesced.
__global__ void pair_pos_kernel(int64_t N, const uint32_t* __restrict__ sorted_pairs, uint32_t* __restrict__ pos)
{
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < 8 * N) {
        const uint32_t s = sorted_pairs[j];
        pos[(int64_t)(s & 7u) * N + (s >> 3)] = (uint32_t)j;
    }
}

}  // namespace svr
