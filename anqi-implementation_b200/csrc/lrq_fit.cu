// LRQ verifier fit on the device (FP64): the rounds of the reference trainer
// (tools/train_final_m8_u8.py:81-258) as kernels, for a host driver that keeps
// only the 100 x 100 eigen-decomposition on the CPU.
//
//   stats     mean and covariance of X = keys[ids] - sub   (fit_basis, :81-89)
//   residual  res = T - (mu + ((T - mu) G^T) G), column-major (reconstruct, :90-93)
//   codebooks per column: sort, prefix sums, 1-D Lloyd from quantile centres
//             with a monotone repair (:97-144)
//   decode    nearest centre per value (decode_nearest, :146-156) and the
//             squared reconstruction error of the round
//   range     per-column min / max of the residuals of all n rows (:159-174)
//
// Orders of summation: the prefix sums run in index order as NumPy's cumsum
// does; the sort is exact; the mean, covariance and reconstruction sum in
// their own (fixed, deterministic) orders, so results agree with the NumPy
// fit to rounding, not bit for bit.  Every entry point takes device pointers,
// enqueues on the caller's stream and allocates nothing; scratch comes from
// the caller with its size checked.
#include <cfloat>

#include "common.cuh"
#include "internal.h"

namespace anqi {
namespace {

constexpr uint32_t kFitMaxCols = 128;  // nk
constexpr uint32_t kFitMaxRank = 16;   // rank M
constexpr uint32_t kStatRows = 1024;   // rows per block of the partial sums
constexpr uint32_t kSortChunk = 2048;  // elements sorted per block in shared memory

__device__ __forceinline__ double row_value(const float* keys, const uint32_t* ids, uint64_t i, uint32_t nk, uint32_t k) {
    const uint64_t r = ids ? (uint64_t)ids[i] : i;
    return (double)keys[r * nk + k];
}

// ---------------------------------------------------------------- stats

// partial[b][k] = sum over the block's rows of X[i,k] (X = keys[ids] - sub)
__global__ void fit_colsum_kernel(const float* __restrict__ keys, const uint32_t* __restrict__ ids, uint64_t m,
                                  uint32_t nk, const double* __restrict__ sub, double* __restrict__ partial) {
    const uint64_t r0 = (uint64_t)blockIdx.x * kStatRows;
    const uint64_t r1 = m < r0 + kStatRows ? m : r0 + kStatRows;
    for (uint32_t k = threadIdx.x; k < nk; k += blockDim.x) {
        double s = 0.0;
        for (uint64_t i = r0; i < r1; i++) {
            const double x = row_value(keys, ids, i, nk, k) - (sub ? sub[(uint64_t)k * m + i] : 0.0);
            s = __dadd_rn(s, x);
        }
        partial[(uint64_t)blockIdx.x * nk + k] = s;
    }
}

// out[j] = sum_b partial[b][j] / m, in block order
__global__ void fit_reduce_kernel(const double* __restrict__ partial, uint32_t nblk, uint32_t width, double scale,
                                  double* __restrict__ out) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < width; j += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (uint32_t b = 0; b < nblk; b++) s = __dadd_rn(s, partial[(uint64_t)b * width + j]);
        out[j] = __dmul_rn(s, scale);
    }
}

// partial[b][k*nk+l] = sum over the block's rows of (X[i,k]-mean[k]) (X[i,l]-mean[l]), k <= l
__global__ void __launch_bounds__(256) fit_cov_kernel(const float* __restrict__ keys, const uint32_t* __restrict__ ids,
                                                      uint64_t m, uint32_t nk, const double* __restrict__ sub,
                                                      const double* __restrict__ mean, double* __restrict__ partial) {
    constexpr uint32_t kRows = 32;
    __shared__ double tile[kRows][kFitMaxCols];
    const uint64_t r0 = (uint64_t)blockIdx.x * kStatRows;
    const uint64_t r1 = m < r0 + kStatRows ? m : r0 + kStatRows;
    const uint32_t npair = nk * (nk + 1) / 2;
    constexpr uint32_t kPer = (kFitMaxCols * (kFitMaxCols + 1) / 2 + 255) / 256;
    double acc[kPer];
    uint32_t pk[kPer], pl[kPer];
#pragma unroll
    for (uint32_t t = 0; t < kPer; t++) {
        acc[t] = 0.0;
        // pair index p -> (k, l), k <= l, row-major over the upper triangle
        uint32_t p = threadIdx.x + t * 256u, k = 0;
        if (p < npair) {
            while (p >= nk - k) {
                p -= nk - k;
                k++;
            }
            pk[t] = k;
            pl[t] = k + p;
        } else {
            pk[t] = pl[t] = 0;
        }
    }
    for (uint64_t b0 = r0; b0 < r1; b0 += kRows) {
        const uint32_t rows = (uint32_t)(r1 - b0 < kRows ? r1 - b0 : kRows);
        __syncthreads();
        for (uint32_t t = threadIdx.x; t < rows * nk; t += blockDim.x) {
            const uint32_t rr = t / nk, k = t % nk;
            const uint64_t i = b0 + rr;
            tile[rr][k] = row_value(keys, ids, i, nk, k) - (sub ? sub[(uint64_t)k * m + i] : 0.0) - mean[k];
        }
        __syncthreads();
#pragma unroll
        for (uint32_t t = 0; t < kPer; t++) {
            if (threadIdx.x + t * 256u >= npair) continue;
            const uint32_t k = pk[t], l = pl[t];
            for (uint32_t rr = 0; rr < rows; rr++) acc[t] = __dadd_rn(acc[t], __dmul_rn(tile[rr][k], tile[rr][l]));
        }
    }
#pragma unroll
    for (uint32_t t = 0; t < kPer; t++) {
        if (threadIdx.x + t * 256u >= npair) continue;
        partial[(uint64_t)blockIdx.x * nk * nk + pk[t] * nk + pl[t]] = acc[t];
        partial[(uint64_t)blockIdx.x * nk * nk + pl[t] * nk + pk[t]] = acc[t];
    }
}

// ------------------------------------------------------------- residual

// One warp per row: c = (T - mu) G^T (a sum over k per rank, lanes over k,
// folded by shuffles), rec = mu + c G, res = T - rec.  Writes column-major.
template <bool kAllRows>
__global__ void __launch_bounds__(256) fit_residual_kernel(const float* __restrict__ keys,
                                                           const uint32_t* __restrict__ ids, uint64_t m, uint32_t nk,
                                                           const double* __restrict__ mu, const double* __restrict__ G,
                                                           uint32_t rank, double* __restrict__ res,
                                                           double* __restrict__ lohi, uint32_t* __restrict__ status) {
    constexpr uint32_t kC = kFitMaxCols / 32;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t w0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    double lo[kC], hi[kC];
#pragma unroll
    for (uint32_t j = 0; j < kC; j++) {
        lo[j] = __longlong_as_double(0x7ff0000000000000ll);
        hi[j] = -lo[j];
    }
    bool bad = false;
    for (uint64_t i = w0; i < m; i += nw) {
        double t[kC], cen[kC];
#pragma unroll
        for (uint32_t j = 0; j < kC; j++) {
            const uint32_t k = lane + 32 * j;
            t[j] = k < nk ? row_value(keys, ids, i, nk, k) : 0.0;
            cen[j] = k < nk ? t[j] - mu[k] : 0.0;
        }
        double c[kFitMaxRank];
#pragma unroll
        for (uint32_t r = 0; r < kFitMaxRank; r++) {
            if (r >= rank) {
                c[r] = 0.0;
                continue;
            }
            double s = 0.0;
#pragma unroll
            for (uint32_t j = 0; j < kC; j++) {
                const uint32_t k = lane + 32 * j;
                if (k < nk) s = __fma_rn(cen[j], G[(uint64_t)r * nk + k], s);
            }
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
            c[r] = s;
        }
#pragma unroll
        for (uint32_t j = 0; j < kC; j++) {
            const uint32_t k = lane + 32 * j;
            if (k >= nk) continue;
            double rec = 0.0;
#pragma unroll
            for (uint32_t r = 0; r < kFitMaxRank; r++)
                if (r < rank) rec = __fma_rn(c[r], G[(uint64_t)r * nk + k], rec);
            const double v = t[j] - (mu[k] + rec);
            bad |= !isfinite(v);
            if (kAllRows) {
                lo[j] = fmin(lo[j], v);
                hi[j] = fmax(hi[j], v);
            } else {
                res[(uint64_t)k * m + i] = v;
            }
        }
    }
    if (bad) atomicOr(status, 1u);
    if (kAllRows) {
        // per-warp min / max, then one atomic per column and block-warp (exact: order-free)
#pragma unroll
        for (uint32_t j = 0; j < kC; j++) {
            const uint32_t k = lane + 32 * j;
            if (k >= nk) continue;
            // doubles as ordered integers: min over the value, max over the value
            const double a = lo[j], b = hi[j];
            unsigned long long* pa = reinterpret_cast<unsigned long long*>(lohi + 2 * k);
            unsigned long long* pb = reinterpret_cast<unsigned long long*>(lohi + 2 * k + 1);
            unsigned long long old = *pa, assumed;
            do {
                assumed = old;
                if (__longlong_as_double((long long)assumed) <= a) break;
                old = atomicCAS(pa, assumed, (unsigned long long)__double_as_longlong(a));
            } while (old != assumed);
            old = *pb;
            do {
                assumed = old;
                if (__longlong_as_double((long long)assumed) >= b) break;
                old = atomicCAS(pb, assumed, (unsigned long long)__double_as_longlong(b));
            } while (old != assumed);
        }
    }
}

__global__ void fit_lohi_init_kernel(double* lohi, uint32_t nk) {
    for (uint32_t k = threadIdx.x; k < nk; k += blockDim.x) {
        lohi[2 * k] = __longlong_as_double(0x7ff0000000000000ll);
        lohi[2 * k + 1] = __longlong_as_double((long long)0xfff0000000000000ull);
    }
}

// ---------------------------------------------------------------- sort

// Copies column k of res (m values) into a padded row of n2 (+inf beyond m).
__global__ void fit_pad_kernel(const double* __restrict__ res, uint64_t m, uint32_t nk, uint64_t n2,
                               double* __restrict__ a) {
    const uint64_t total = (uint64_t)nk * n2;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = t / n2, i = t % n2;
        a[t] = i < m ? res[k * m + i] : __longlong_as_double(0x7ff0000000000000ll);
    }
}

// Bitonic stages (kk, j) with j >= kSortChunk: one compare-exchange per thread.
__global__ void fit_bitonic_global_kernel(double* __restrict__ a, uint64_t total, uint64_t n2, uint64_t kk,
                                          uint64_t j) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total / 2;
         t += (uint64_t)gridDim.x * blockDim.x) {
        // the t-th pair: i has bit j clear
        const uint64_t i = (t / j) * 2 * j + (t % j);
        const uint64_t p = i + j;
        const uint64_t pos = i % n2;  // position within the column
        const bool up = (pos & kk) == 0;
        const double x = a[i], y = a[p];
        if ((x > y) == up) {
            a[i] = y;
            a[p] = x;
        }
    }
}

// Bitonic stages j < kSortChunk for every kk in [kk_lo, kk_hi] inside chunks
// of kSortChunk elements held in shared memory.
__global__ void __launch_bounds__(1024) fit_bitonic_shared_kernel(double* __restrict__ a, uint64_t n2, uint64_t kk_lo,
                                                                  uint64_t kk_hi) {
    __shared__ double s[kSortChunk];
    const uint64_t base = (uint64_t)blockIdx.x * kSortChunk;
    for (uint32_t t = threadIdx.x; t < kSortChunk; t += blockDim.x) s[t] = a[base + t];
    __syncthreads();
    for (uint64_t kk = kk_lo; kk <= kk_hi; kk <<= 1) {
        for (uint64_t j = (kk >> 1) < (kSortChunk >> 1) ? (kk >> 1) : (kSortChunk >> 1); j > 0; j >>= 1) {
            for (uint32_t t = threadIdx.x; t < kSortChunk / 2; t += blockDim.x) {
                const uint32_t i = (uint32_t)((t / j) * 2 * j + (t % j));
                const uint32_t p = i + (uint32_t)j;
                const bool up = (((base + i) % n2) & kk) == 0;
                const double x = s[i], y = s[p];
                if ((x > y) == up) {
                    s[i] = y;
                    s[p] = x;
                }
            }
            __syncthreads();
        }
    }
    for (uint32_t t = threadIdx.x; t < kSortChunk; t += blockDim.x) a[base + t] = s[t];
}

// prefix[k][0] = 0, prefix[k][i+1] = prefix[k][i] + s[k][i], in index order (np.cumsum)
__global__ void fit_prefix_kernel(const double* __restrict__ a, uint64_t m, uint32_t nk, uint64_t n2,
                                  double* __restrict__ prefix) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nk) return;
    const double* s = a + (uint64_t)k * n2;
    double* pf = prefix + (uint64_t)k * (m + 1);
    double run = 0.0;
    pf[0] = 0.0;
    for (uint64_t i = 0; i < m; i++) {
        run = __dadd_rn(run, s[i]);
        pf[i + 1] = run;
    }
}

// ---------------------------------------------------------------- Lloyd

// first index with s[i] > v (np.searchsorted side="right")
__device__ __forceinline__ uint64_t search_right(const double* s, uint64_t m, double v) {
    uint64_t lo = 0, hi = m;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (s[mid] <= v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// One block per column, one thread per centre (cs <= blockDim.x).
__global__ void __launch_bounds__(256) fit_lloyd_kernel(const double* __restrict__ a, uint64_t m, uint64_t n2,
                                                        const double* __restrict__ prefix, uint32_t cs, uint32_t iters,
                                                        double* __restrict__ codebooks) {
    __shared__ double cen[256], upd[256];
    __shared__ uint64_t cut[256];
    __shared__ int s_done;
    const uint32_t k = blockIdx.x, c = threadIdx.x;
    const double* s = a + (uint64_t)k * n2;
    const double* pf = prefix + (uint64_t)k * (m + 1);
    double* out = codebooks + (uint64_t)k * cs;
    if (s[0] == s[m - 1]) {
        if (c < cs) out[c] = s[0];
        return;
    }
    if (c < cs) {
        // np.quantile, method "linear": virtual index n q + (1 - q) - 1, then
        // the lerp a + (b - a) t (b - (b - a)(1 - t) when t >= 0.5)
        const double q = ((double)c + 0.5) / (double)cs;
        const double vi = __dsub_rn(__dadd_rn(__dmul_rn((double)m, q), __dadd_rn(1.0, __dmul_rn(q, -1.0))), 1.0);
        double fl = floor(vi);
        const double last = (double)(m - 1);
        if (fl < 0.0) fl = 0.0;
        if (fl > last) fl = last;
        const uint64_t i0 = (uint64_t)fl, i1 = i0 + 1 < m ? i0 + 1 : m - 1;
        const double t = vi - fl;
        const double x0 = s[i0], x1 = s[i1], diff = x1 - x0;
        cen[c] = t >= 0.5 ? __dsub_rn(x1, __dmul_rn(diff, 1.0 - t)) : __dadd_rn(x0, __dmul_rn(diff, t));
    }
    __syncthreads();
    for (uint32_t it = 0; it < iters; it++) {
        if (c + 1 < cs) cut[c] = search_right(s, m, (cen[c] + cen[c + 1]) * 0.5);
        __syncthreads();
        if (c < cs) {
            const uint64_t lo = c == 0 ? 0 : cut[c - 1];
            const uint64_t hi = c + 1 < cs ? cut[c] : m;
            const uint64_t cnt = hi - lo;
            upd[c] = cnt > 0 ? (pf[hi] - pf[lo]) / (double)cnt : cen[c];
        }
        __syncthreads();
        // np.maximum.accumulate: an inclusive max-scan (exact in any order)
        for (uint32_t off = 1; off < cs; off <<= 1) {
            double v = 0.0;
            if (c < cs && c >= off) v = fmax(upd[c], upd[c - off]);
            __syncthreads();
            if (c < cs && c >= off) upd[c] = v;
            __syncthreads();
        }
        if (c == 0) s_done = 1;
        __syncthreads();
        if (c < cs && !(fabs(upd[c] - cen[c]) < 1e-12)) s_done = 0;
        __syncthreads();
        const int done = s_done;
        if (c < cs) cen[c] = upd[c];
        __syncthreads();
        if (done) break;
    }
    if (c < cs) out[c] = cen[c];
}

// ---------------------------------------------------------------- decode

// dec[k][i] = the nearest centre of res[k][i] (lower on ties); partial[b] = the
// block's sum of (dec - res)^2.
__global__ void __launch_bounds__(256) fit_decode_kernel(const double* __restrict__ res, uint64_t m, uint32_t nk,
                                                         const double* __restrict__ codebooks, uint32_t cs,
                                                         double* __restrict__ dec, double* __restrict__ partial) {
    __shared__ double red[256];
    double acc = 0.0;
    const uint64_t total = (uint64_t)nk * m;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = t / m;
        const double v = res[t];
        const double* cb = codebooks + k * cs;
        uint32_t lo = 0, hi = cs;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (cb[mid] < v) lo = mid + 1;
            else hi = mid;
        }
        const uint32_t up = lo < cs ? lo : cs - 1, dn = lo > 0 ? lo - 1 : 0;
        const double d = fabs(cb[up] - v) < fabs(v - cb[dn]) ? cb[up] : cb[dn];
        dec[t] = d;
        acc += (d - v) * (d - v);
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (uint32_t o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

uint32_t grid_for(uint64_t work, uint32_t threads, uint32_t cap = 4096) {
    const uint64_t g = (work + threads - 1) / threads;
    return (uint32_t)(g < 1 ? 1 : (g > cap ? cap : g));
}

}  // namespace
}  // namespace anqi

using namespace anqi;

extern "C" {

int anqi_lrq_fit_stats(const float* keys, const uint32_t* ids, uint64_t m, uint32_t nk, const double* sub,
                       double* scratch, uint64_t scratch_doubles, double* mean, double* cov, void* stream) {
    if (!keys || !scratch || !mean || !cov || m == 0 || nk == 0 || nk > kFitMaxCols) return ANQI_ERR_ARGS;
    const uint32_t nblk = (uint32_t)((m + kStatRows - 1) / kStatRows);
    if (scratch_doubles < (uint64_t)nblk * nk * nk) return ANQI_ERR_CAPACITY;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    fit_colsum_kernel<<<nblk, 128, 0, st>>>(keys, ids, m, nk, sub, scratch);
    fit_reduce_kernel<<<1, 128, 0, st>>>(scratch, nblk, nk, 1.0 / (double)m, mean);
    fit_cov_kernel<<<nblk, 256, 0, st>>>(keys, ids, m, nk, sub, mean, scratch);
    fit_reduce_kernel<<<grid_for((uint64_t)nk * nk, 256), 256, 0, st>>>(scratch, nblk, nk * nk, 1.0 / (double)m, cov);
    return cudaGetLastError() == cudaSuccess ? ANQI_OK : ANQI_ERR_DEVICE;
}

int anqi_lrq_fit_residual(const float* keys, const uint32_t* ids, uint64_t m, uint32_t nk, const double* mu,
                          const double* basis, uint32_t rank, double* res, uint32_t* status, void* stream) {
    if (!keys || !mu || !basis || !res || !status || m == 0 || nk == 0 || nk > kFitMaxCols || rank == 0 ||
        rank > kFitMaxRank)
        return ANQI_ERR_ARGS;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    fit_residual_kernel<false><<<grid_for(m * 32, 256), 256, 0, st>>>(keys, ids, m, nk, mu, basis, rank, res, nullptr,
                                                                      status);
    return cudaGetLastError() == cudaSuccess ? ANQI_OK : ANQI_ERR_DEVICE;
}

int anqi_lrq_fit_range(const float* keys, uint64_t n, uint32_t nk, const double* mu, const double* basis,
                       uint32_t rank, double* lohi, uint32_t* status, void* stream) {
    if (!keys || !mu || !basis || !lohi || !status || n == 0 || nk == 0 || nk > kFitMaxCols || rank == 0 ||
        rank > kFitMaxRank)
        return ANQI_ERR_ARGS;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    fit_lohi_init_kernel<<<1, 128, 0, st>>>(lohi, nk);
    fit_residual_kernel<true><<<grid_for(n * 32, 256, 2048), 256, 0, st>>>(keys, nullptr, n, nk, mu, basis, rank,
                                                                           nullptr, lohi, status);
    return cudaGetLastError() == cudaSuccess ? ANQI_OK : ANQI_ERR_DEVICE;
}

uint64_t anqi_lrq_fit_codebooks_scratch(uint64_t m, uint32_t nk) {
    uint64_t n2 = kSortChunk;
    while (n2 < m) n2 <<= 1;
    return (uint64_t)nk * n2 + (uint64_t)nk * (m + 1);
}

int anqi_lrq_fit_codebooks(const double* res, uint64_t m, uint32_t nk, uint32_t cs, uint32_t iters, double* scratch,
                           uint64_t scratch_doubles, double* codebooks, void* stream) {
    if (!res || !scratch || !codebooks || m < 2 || nk == 0 || nk > kFitMaxCols || cs < 2 || cs > 256)
        return ANQI_ERR_ARGS;
    if (scratch_doubles < anqi_lrq_fit_codebooks_scratch(m, nk)) return ANQI_ERR_CAPACITY;
    uint64_t n2 = kSortChunk;
    while (n2 < m) n2 <<= 1;
    double* a = scratch;
    double* prefix = scratch + (uint64_t)nk * n2;
    const uint64_t total = (uint64_t)nk * n2;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    fit_pad_kernel<<<grid_for(total, 256), 256, 0, st>>>(res, m, nk, n2, a);
    const uint32_t chunks = (uint32_t)(total / kSortChunk);
    // every chunk sorted up to size kSortChunk, then the larger merges
    fit_bitonic_shared_kernel<<<chunks, 1024, 0, st>>>(a, n2, 2, kSortChunk);
    for (uint64_t kk = 2 * kSortChunk; kk <= n2; kk <<= 1) {
        for (uint64_t j = kk >> 1; j >= kSortChunk; j >>= 1)
            fit_bitonic_global_kernel<<<grid_for(total / 2, 256), 256, 0, st>>>(a, total, n2, kk, j);
        fit_bitonic_shared_kernel<<<chunks, 1024, 0, st>>>(a, n2, kk, kk);
    }
    fit_prefix_kernel<<<(nk + 31) / 32, 32, 0, st>>>(a, m, nk, n2, prefix);
    fit_lloyd_kernel<<<nk, 256, 0, st>>>(a, m, n2, prefix, cs, iters, codebooks);
    return cudaGetLastError() == cudaSuccess ? ANQI_OK : ANQI_ERR_DEVICE;
}

int anqi_lrq_fit_decode(const double* res, uint64_t m, uint32_t nk, const double* codebooks, uint32_t cs, double* dec,
                        double* partial, uint32_t partial_cap, uint32_t* n_partial, void* stream) {
    if (!res || !codebooks || !dec || !partial || !n_partial || m == 0 || nk == 0 || cs == 0 || cs > 256)
        return ANQI_ERR_ARGS;
    const uint32_t g = grid_for((uint64_t)nk * m, 256, 1024);
    if (partial_cap < g) return ANQI_ERR_CAPACITY;
    *n_partial = g;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    fit_decode_kernel<<<g, 256, 0, st>>>(res, m, nk, codebooks, cs, dec, partial);
    return cudaGetLastError() == cudaSuccess ? ANQI_OK : ANQI_ERR_DEVICE;
}

}  // extern "C"
