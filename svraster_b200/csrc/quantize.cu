// 8-bit codebook of a saved checkpoint (src/sparse_voxel_gears/io.py:109-170).
//
// Behaviour of io.py:123-167 (quantization): 257 quantiles of the sorted values (float32
// positions j/256 * (n-1), truncated; entry 0 replaced by -inf), a left searchsorted, the
// nearer of the two candidate entries (index -1 reads entry 255, torch's negative index), then
// up to max_iter rounds of (per-entry mean, move each value one entry towards a strictly
// nearer neighbour) stopping at the first round that moves nothing, and a final mean; entries
// that hold no value are 0.  Organisation (ours): one radix sort for the quantiles; the
// assignment and every round are one pass each that also accumulates the next round's
// per-entry sums (float64, block-local in shared memory, then one atomic per entry and block);
// the index array doubles as the output.  The reference's means are float32 sums in its
// thread or value order; the float64 sums here round to the correctly rounded mean in all
// but rare cases, so codebooks agree to float32 rounding and indices wherever a value is not
// within that rounding of the midpoint of two entries.
#include <cstdint>
#include <string>

#include <cub/device/device_radix_sort.cuh>

#include "svr_common.cuh"

using namespace svr;

int svr_fail(int code, const char* what);
void svr_note_launch(int n);

#define CUDA_TRY(x)                                                                      \
    do {                                                                                 \
        cudaError_t e_ = (x);                                                            \
        if (e_ != cudaSuccess) {                                                         \
            return svr_fail(SVR_ERR_CUDA, (std::string(#x) + ": " + cudaGetErrorString(e_)).c_str()); \
        }                                                                                \
    } while (0)
#define LAUNCHED() do { svr_note_launch(1); CUDA_TRY(cudaGetLastError()); } while (0)

static inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

namespace {

constexpr int NB = 256;          // codebook entries
constexpr int QT = 256;          // threads per block of the element passes
constexpr unsigned ERR_NONFINITE = 32u;

struct Acc {                     // per-entry sums of the next mean, and the moved count
    double sum[NB];
    unsigned long long cnt[NB];
    unsigned long long moved;
};

struct QuantWs {
    size_t sorted, full, acc, tmp, tmp_bytes, total;
};

int quant_ws(int64_t n, QuantWs& w)
{
    w.sorted = 0;
    w.full = align_up(4 * (size_t)n, 256);
    w.acc = w.full + align_up(4 * 257, 256);
    w.tmp = w.acc + align_up(sizeof(Acc), 256);
    w.tmp_bytes = 0;
    cudaError_t e = cub::DeviceRadixSort::SortKeys(nullptr, w.tmp_bytes, (const float*)nullptr, (float*)nullptr,
                                                   (int)n);
    if (e != cudaSuccess) return svr_fail(SVR_ERR_CUDA, "quantize: sort size query");
    w.total = align_up(w.tmp + w.tmp_bytes, 256);
    return SVR_OK;
}

__global__ void quant_init_kernel(int64_t n, const float* __restrict__ sorted, float* __restrict__ full,
                                  Acc* __restrict__ acc)
{
    const int j = threadIdx.x;
    if (j < 257) {
        // torch.linspace(0, 1, 257)[j] is j / 256 exactly; the product is one float32 multiply
        const float pos = __fmul_rn((float)j * (1.0f / 256.0f), (float)(n - 1));
        long long q = (long long)pos;
        q = q < 0 ? 0 : (q > n - 1 ? n - 1 : q);
        full[j] = j == 0 ? -INFINITY : sorted[q];
    }
    if (j < NB) { acc->sum[j] = 0.0; acc->cnt[j] = 0ull; }
    if (j == 0) acc->moved = 0ull;
}

__device__ __forceinline__ void acc_block(double* ssum, unsigned* scnt, int k, float x)
{
    atomicAdd(ssum + k, (double)x);
    atomicAdd(scnt + k, 1u);
}

__device__ __forceinline__ void acc_flush(const double* ssum, const unsigned* scnt, Acc* acc)
{
    for (int b = threadIdx.x; b < NB; b += blockDim.x)
        if (scnt[b]) {
            atomicAdd(acc->sum + b, ssum[b]);
            atomicAdd(acc->cnt + b, (unsigned long long)scnt[b]);
        }
}

__global__ void __launch_bounds__(QT) quant_assign_kernel(int64_t n, const float* __restrict__ v,
                                                          const float* __restrict__ full,
                                                          uint8_t* __restrict__ index, Acc* __restrict__ acc,
                                                          unsigned* status)
{
    __shared__ float sfull[257];
    __shared__ double ssum[NB];
    __shared__ unsigned scnt[NB];
    for (int j = threadIdx.x; j < 257; j += blockDim.x) sfull[j] = full[j];
    for (int b = threadIdx.x; b < NB; b += blockDim.x) { ssum[b] = 0.0; scnt[b] = 0u; }
    __syncthreads();
    const float* cb = sfull + 1;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float x = v[i];
        if (!isfinite(x)) atomicOr(status, ERR_NONFINITE);
        int lo = 0, hi = 257;                      // first entry >= x
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (sfull[mid] < x) lo = mid + 1; else hi = mid;
        }
        int k = min(max(lo - 1, 0), NB - 1);
        const float dl = fabsf(x - cb[k == 0 ? NB - 1 : k - 1]), dm = fabsf(x - cb[k]);
        k = min(max(k - 1 + (dm < dl ? 1 : 0), 0), NB - 1);
        index[i] = (uint8_t)k;
        acc_block(ssum, scnt, k, x);
    }
    __syncthreads();
    acc_flush(ssum, scnt, acc);
}

// book = the accumulated means; the accumulator is cleared for the next pass
__global__ void quant_mean_kernel(Acc* __restrict__ acc, float* __restrict__ book)
{
    const int b = threadIdx.x;
    if (b < NB) {
        const unsigned long long c = acc->cnt[b];
        book[b] = c ? (float)(acc->sum[b] / (double)c) : 0.f;
        acc->sum[b] = 0.0;
        acc->cnt[b] = 0ull;
    }
    if (b == 0) acc->moved = 0ull;
}

__global__ void __launch_bounds__(QT) quant_round_kernel(int64_t n, const float* __restrict__ v,
                                                         const float* __restrict__ book,
                                                         uint8_t* __restrict__ index, Acc* __restrict__ acc)
{
    __shared__ float sbook[NB];
    __shared__ double ssum[NB];
    __shared__ unsigned scnt[NB];
    __shared__ unsigned smoved;
    for (int b = threadIdx.x; b < NB; b += blockDim.x) { sbook[b] = book[b]; ssum[b] = 0.0; scnt[b] = 0u; }
    if (threadIdx.x == 0) smoved = 0u;
    __syncthreads();
    unsigned moved = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float x = v[i];
        int k = index[i];
        const float dl = fabsf(x - sbook[k == 0 ? NB - 1 : k - 1]);
        const float dr = fabsf(x - sbook[k == NB - 1 ? NB - 1 : k + 1]);
        const float dm = fabsf(x - sbook[k]);
        if (fminf(dl, dr) < dm) {
            k = min(max(k + (dr < dl ? 1 : -1), 0), NB - 1);
            index[i] = (uint8_t)k;
            ++moved;
        }
        acc_block(ssum, scnt, k, x);
    }
    moved = __reduce_add_sync(0xffffffffu, moved);
    if ((threadIdx.x & 31) == 0 && moved) atomicAdd(&smoved, moved);
    __syncthreads();
    acc_flush(ssum, scnt, acc);
    if (threadIdx.x == 0 && smoved) atomicAdd(&acc->moved, (unsigned long long)smoved);
}

__global__ void dequant_kernel(int64_t n, const uint8_t* __restrict__ index, const float* __restrict__ book,
                               float* __restrict__ out)
{
    __shared__ float sbook[NB];
    for (int b = threadIdx.x; b < NB; b += blockDim.x) sbook[b] = book[b];
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = sbook[index[i]];
}

unsigned grid_for(int64_t n)
{
    // enough blocks for 8 per SM on 148 SMs, fewer for small inputs
    const int64_t want = (n + QT - 1) / QT;
    return (unsigned)(want < 148 * 8 ? (want > 0 ? want : 1) : 148 * 8);
}

}  // namespace

extern "C" int svr_quantize_workspace_bytes(int64_t n, size_t* bytes)
{
    if (!bytes || n <= 0 || n >= (1ll << 31)) return svr_fail(SVR_ERR_ARG, "quantize: n must be in [1, 2^31)");
    QuantWs w;
    if (int rc = quant_ws(n, w)) return rc;
    *bytes = w.total;
    return SVR_OK;
}

extern "C" int svr_quantize(int64_t n, const float* values, int max_iter, uint8_t* index_out, float* codebook_out,
                            void* ws, size_t ws_bytes, int* rounds_host, uint32_t* status, void* stream)
{
    size_t need = 0;
    if (int rc = svr_quantize_workspace_bytes(n, &need)) return rc;
    if (!values || !index_out || !codebook_out || !status || !ws || ws_bytes < need || max_iter < 0)
        return svr_fail(SVR_ERR_ARG, "quantize: bad argument or workspace too small");
    QuantWs w;
    if (int rc = quant_ws(n, w)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    char* base = (char*)ws;
    float* sorted = (float*)(base + w.sorted);
    float* full = (float*)(base + w.full);
    Acc* acc = (Acc*)(base + w.acc);
    size_t tb = w.tmp_bytes;
    CUDA_TRY(cub::DeviceRadixSort::SortKeys(base + w.tmp, tb, values, sorted, (int)n, 0, 32, st));
    quant_init_kernel<<<1, 288, 0, st>>>(n, sorted, full, acc);
    LAUNCHED();
    const unsigned g = grid_for(n);
    quant_assign_kernel<<<g, QT, 0, st>>>(n, values, full, index_out, acc, status);
    LAUNCHED();
    int rounds = 0;
    for (int it = 0; it < max_iter; ++it) {
        quant_mean_kernel<<<1, NB, 0, st>>>(acc, codebook_out);
        LAUNCHED();
        quant_round_kernel<<<g, QT, 0, st>>>(n, values, codebook_out, index_out, acc);
        LAUNCHED();
        unsigned long long moved = 0;
        CUDA_TRY(cudaMemcpyAsync(&moved, &acc->moved, sizeof(moved), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        if (moved == 0) break;     // nothing moved: the accumulator holds the same means again
        ++rounds;
    }
    quant_mean_kernel<<<1, NB, 0, st>>>(acc, codebook_out);
    LAUNCHED();
    if (rounds_host) *rounds_host = rounds;
    return SVR_OK;
}

extern "C" int svr_dequantize(int64_t n, const uint8_t* index, const float* codebook, float* out, void* stream)
{
    if (n <= 0) return n == 0 ? SVR_OK : svr_fail(SVR_ERR_ARG, "dequantize: n");
    if (!index || !codebook || !out) return svr_fail(SVR_ERR_ARG, "dequantize: null argument");
    dequant_kernel<<<grid_for(n), QT, 0, (cudaStream_t)stream>>>(n, index, codebook, out);
    LAUNCHED();
    return SVR_OK;
}
