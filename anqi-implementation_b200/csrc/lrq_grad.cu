// LRQ radius-reconstruction objective: CUDA forward and backward (FP64).
//
// The quantity the reference trainer's rounds minimise
// (tools/train_final_m8_u8.py:90-157, 206-218): for cutoff rows T (n x nk),
// mean mu (nk), rank-M basis G (m x nk) and per-rank codebook B (nk x cs,
// rows ascending),
//   c[o,:]  = (T[o,:] - mu) G^T                    (reconstruct, :90-93)
//   base    = mu + c G
//   a[o,k]  = decode_nearest(T - base)             (:146-156: the insertion
//             point of the value in row k, then the closer of the two
//             neighbours, the lower one on ties)
//   r       = base + B[k, a] - T
//   loss    = sum(r^2) / (n nk)
// With the codes held fixed (a is piecewise constant in the parameters):
//   dL/dB[k,j] = 2/(n nk) sum_{o: a[o,k]=j} r[o,k]
//   dL/dmu[k]  = 2/(n nk) sum_o (r[o,k] - sum_m G[m,k] s[o,m]),  s = r G^T
//   dL/dG[m,k] = 2/(n nk) sum_o (r[o,k] c[o,m] + (T[o,k] - mu[k]) s[o,m])
//
// One warp per row, lanes over the nk columns.  Entry points take device
// pointers and a stream and allocate nothing.
#include "common.cuh"
#include "internal.h"

namespace anqi {
namespace {

constexpr uint32_t kMaxCols = 4;  // per-lane columns: nk <= 128
constexpr unsigned kWarp = 0xFFFFFFFFu;

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kWarp, v, o);
    return v;
}

// decode_nearest on one ascending codebook row.
__device__ __forceinline__ uint32_t nearest_code(const double* __restrict__ row, uint32_t cs, double v) {
    uint32_t lo = 0, hi = cs;  // first index with row[i] >= v
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (row[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    const uint32_t high = lo < cs ? lo : cs - 1;
    const uint32_t low = lo > 0 ? lo - 1 : 0;
    return fabs(row[high] - v) < fabs(v - row[low]) ? high : low;
}

struct ObjParams {
    const double* T;
    uint64_t n;
    uint32_t nk, m, cs;
    const double* mu;
    const double* G;
    const double* B;
    const uint8_t* codes_in;  // optional: use these codes instead of the nearest ones
    double* r;
    double* c;
    uint8_t* a;
    double* loss;             // one accumulator, zeroed by the host
};

// M: compile-time bound on the rank (m <= M), so per-rank values stay in registers.
template <uint32_t M>
__global__ void lrq_objective_forward_kernel(ObjParams p) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    double part = 0.0;
    for (uint64_t o = w; o < p.n; o += nw) {
        const double* t = p.T + o * p.nk;
        double tv[kMaxCols], cen[kMaxCols];
#pragma unroll
        for (uint32_t j = 0; j < kMaxCols; j++) {
            const uint32_t k = lane + 32 * j;
            tv[j] = k < p.nk ? t[k] : 0.0;
            cen[j] = k < p.nk ? tv[j] - p.mu[k] : 0.0;
        }
        double cm[M];
#pragma unroll
        for (uint32_t mm = 0; mm < M; mm++) {
            cm[mm] = 0.0;
            if (mm >= p.m) continue;
            double s = 0.0;
#pragma unroll
            for (uint32_t j = 0; j < kMaxCols; j++) {
                const uint32_t k = lane + 32 * j;
                if (k < p.nk) s = fma(cen[j], p.G[(size_t)mm * p.nk + k], s);
            }
            cm[mm] = warp_sum(s);
            if (lane == 0) p.c[o * p.m + mm] = cm[mm];
        }
#pragma unroll
        for (uint32_t j = 0; j < kMaxCols; j++) {
            const uint32_t k = lane + 32 * j;
            if (k >= p.nk) continue;
            double base = p.mu[k];
#pragma unroll
            for (uint32_t mm = 0; mm < M; mm++)
                if (mm < p.m) base = fma(cm[mm], p.G[(size_t)mm * p.nk + k], base);
            const double* row = p.B + (size_t)k * p.cs;
            const uint32_t code =
                p.codes_in ? min((uint32_t)p.codes_in[o * p.nk + k], p.cs - 1) : nearest_code(row, p.cs, tv[j] - base);
            const double rv = base + row[code] - tv[j];
            p.r[o * p.nk + k] = rv;
            p.a[o * p.nk + k] = (uint8_t)code;
            part = fma(rv, rv, part);
        }
    }
    part = warp_sum(part);
    if (lane == 0) atomicAdd(p.loss, part);
}

struct GradParams {
    const double* T;
    uint64_t n;
    uint32_t nk, m, cs;
    const double* mu;
    const double* G;
    const double* r;
    const double* c;
    const uint8_t* a;
    double scale;  // dL/d(sum r^2) times the incoming gradient
    double* g_mu;
    double* g_G;
    double* g_B;
};

template <uint32_t M>
__global__ void lrq_objective_backward_kernel(GradParams p) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    double gmu[kMaxCols] = {0, 0, 0, 0};
    double gG[M][kMaxCols];
#pragma unroll
    for (uint32_t mm = 0; mm < M; mm++)
#pragma unroll
        for (uint32_t j = 0; j < kMaxCols; j++) gG[mm][j] = 0.0;
    for (uint64_t o = w; o < p.n; o += nw) {
        double rv[kMaxCols], cen[kMaxCols];
#pragma unroll
        for (uint32_t j = 0; j < kMaxCols; j++) {
            const uint32_t k = lane + 32 * j;
            rv[j] = k < p.nk ? p.r[o * p.nk + k] : 0.0;
            cen[j] = k < p.nk ? p.T[o * p.nk + k] - p.mu[k] : 0.0;
            if (k < p.nk) atomicAdd(p.g_B + (size_t)k * p.cs + p.a[o * p.nk + k], p.scale * rv[j]);
        }
#pragma unroll
        for (uint32_t mm = 0; mm < M; mm++) {
            if (mm >= p.m) continue;
            double s = 0.0;
#pragma unroll
            for (uint32_t j = 0; j < kMaxCols; j++) {
                const uint32_t k = lane + 32 * j;
                if (k < p.nk) s = fma(p.G[(size_t)mm * p.nk + k], rv[j], s);
            }
            s = warp_sum(s);
            const double cm = p.c[o * p.m + mm];
#pragma unroll
            for (uint32_t j = 0; j < kMaxCols; j++) {
                const uint32_t k = lane + 32 * j;
                if (k >= p.nk) continue;
                gmu[j] = fma(-p.G[(size_t)mm * p.nk + k], s, gmu[j]);
                gG[mm][j] = fma(rv[j], cm, fma(cen[j], s, gG[mm][j]));
            }
        }
#pragma unroll
        for (uint32_t j = 0; j < kMaxCols; j++) gmu[j] += rv[j];
    }
#pragma unroll
    for (uint32_t j = 0; j < kMaxCols; j++) {
        const uint32_t k = lane + 32 * j;
        if (k >= p.nk) continue;
        atomicAdd(p.g_mu + k, p.scale * gmu[j]);
#pragma unroll
        for (uint32_t mm = 0; mm < M; mm++)
            if (mm < p.m) atomicAdd(p.g_G + (size_t)mm * p.nk + k, p.scale * gG[mm][j]);
    }
}

// One warp per row, 8 warps per block, at most 8 blocks per SM (grid-stride).
int launch_grid(uint64_t rows) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (int)std::min<uint64_t>((rows + 7) / 8, (uint64_t)sms * 8);
}

}  // namespace
}  // namespace anqi

using namespace anqi;

extern "C" {

int anqi_lrq_objective_forward(const double* T, uint64_t n, uint32_t nk, uint32_t m, const double* mu,
                               const double* G, const double* B, uint32_t cs, const uint8_t* codes_in, double* r,
                               double* c, uint8_t* a, double* loss, void* stream) {
    if (!T || !mu || !G || !B || !r || !c || !a || !loss || n == 0) return ANQI_ERR_ARGS;
    if (nk == 0 || nk > 32 * kMaxCols || m == 0 || m > 16 || cs == 0 || cs > 256) return ANQI_ERR_ARGS;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(loss, 0, sizeof(double), st) != cudaSuccess) return ANQI_ERR_DEVICE;
    ObjParams p{T, n, nk, m, cs, mu, G, B, codes_in, r, c, a, loss};
    if (m <= 8) lrq_objective_forward_kernel<8><<<launch_grid(n), 256, 0, st>>>(p);
    else lrq_objective_forward_kernel<16><<<launch_grid(n), 256, 0, st>>>(p);
    return cudaGetLastError() == cudaSuccess ? ANQI_OK : ANQI_ERR_DEVICE;
}

int anqi_lrq_objective_backward(const double* T, uint64_t n, uint32_t nk, uint32_t m, const double* mu,
                                const double* G, const double* r, const double* c, const uint8_t* a, uint32_t cs,
                                double scale, double* g_mu, double* g_G, double* g_B, void* stream) {
    if (!T || !mu || !G || !r || !c || !a || !g_mu || !g_G || !g_B || n == 0) return ANQI_ERR_ARGS;
    if (nk == 0 || nk > 32 * kMaxCols || m == 0 || m > 16 || cs == 0 || cs > 256) return ANQI_ERR_ARGS;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(g_mu, 0, nk * sizeof(double), st) != cudaSuccess ||
        cudaMemsetAsync(g_G, 0, (size_t)m * nk * sizeof(double), st) != cudaSuccess ||
        cudaMemsetAsync(g_B, 0, (size_t)nk * cs * sizeof(double), st) != cudaSuccess)
        return ANQI_ERR_DEVICE;
    GradParams p{T, n, nk, m, cs, mu, G, r, c, a, scale, g_mu, g_G, g_B};
    if (m <= 8) lrq_objective_backward_kernel<8><<<launch_grid(n), 256, 0, st>>>(p);
    else lrq_objective_backward_kernel<16><<<launch_grid(n), 256, 0, st>>>(p);
    return cudaGetLastError() == cudaSuccess ? ANQI_OK : ANQI_ERR_DEVICE;
}

}  // extern "C"
