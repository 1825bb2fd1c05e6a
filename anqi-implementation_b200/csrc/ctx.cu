#include <algorithm>
// Context lifetime, device memory, error reporting, and small shared kernels.
#include <cstdarg>
#include <cstdio>
#include <thread>

#include "common.cuh"
#include "internal.h"

namespace anqi {

int fail(Ctx* c, int status, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->last_error = buf;
    return status;
}

int cuda_check(Ctx* c, cudaError_t e, const char* what) {
    return fail(c, ANQI_ERR_DEVICE, "CUDA error in %s: %s", what, cudaGetErrorString(e));
}

int ensure(Ctx* c, DevBuf& b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.bytes >= bytes) return ANQI_OK;
    if (b.p) {
        cudaFree(b.p);
        c->device_bytes -= b.bytes;
        b.p = nullptr;
        b.bytes = 0;
    }
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) {
        b.p = nullptr;
        return fail(c, ANQI_ERR_DEVICE, "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
    }
    b.bytes = bytes;
    c->device_bytes += bytes;
    return ANQI_OK;
}

void release(Ctx* c, DevBuf& b) {
    if (b.p) {
        cudaFree(b.p);
        c->device_bytes -= b.bytes;
    }
    b.p = nullptr;
    b.bytes = 0;
}

// Large copies between pageable host memory and the device go through the
// context's pinned staging slots: host threads copy one chunk into (or out of)
// a slot while the copy engine moves another, instead of the driver staging
// pageable memory through one thread.  Pinned or registered host memory and
// small copies go direct.
constexpr size_t kStageChunk = (size_t)32 << 20;
constexpr size_t kStageMin = (size_t)48 << 20;

static void par_memcpy(void* dst, const void* src, size_t bytes) {
    const unsigned hw = std::thread::hardware_concurrency();
    const unsigned T = std::max(1u, std::min(8u, hw / 2));
    const size_t part = ((bytes + T - 1) / T + 4095) & ~(size_t)4095;
    if (T == 1 || bytes < ((size_t)4 << 20)) {
        std::memcpy(dst, src, bytes);
        return;
    }
    std::vector<std::thread> th;
    for (unsigned t = 1; t < T && (size_t)t * part < bytes; t++) {
        const size_t o = (size_t)t * part, len = std::min(part, bytes - o);
        th.emplace_back([=] { std::memcpy(static_cast<char*>(dst) + o, static_cast<const char*>(src) + o, len); });
    }
    std::memcpy(dst, src, std::min(part, bytes));
    for (std::thread& x : th) x.join();
}

static bool staged(Ctx* c, const void* host, size_t bytes) {
    if (bytes < kStageMin) return false;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, host) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type != cudaMemoryTypeUnregistered) return false;
    if (!c->stage[0]) {
        for (int s = 0; s < Ctx::kStageSlots; s++) {
            if (cudaHostAlloc(&c->stage[s], kStageChunk, cudaHostAllocDefault) != cudaSuccess ||
                cudaEventCreateWithFlags(&c->stage_ev[s], cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                for (int t = 0; t <= s; t++) {
                    if (c->stage[t]) cudaFreeHost(c->stage[t]);
                    if (c->stage_ev[t]) cudaEventDestroy(c->stage_ev[t]);
                    c->stage[t] = nullptr;
                    c->stage_ev[t] = nullptr;
                }
                return false;
            }
        }
    }
    return true;
}

int h2d_raw(Ctx* c, void* dst, const void* src, size_t bytes) {
    if (!bytes) return ANQI_OK;
    if (!staged(c, src, bytes)) {
        ANQI_CUDA(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream));
        return ANQI_OK;
    }
    size_t k = 0;
    for (size_t o = 0; o < bytes; o += kStageChunk, k++) {
        const int s = (int)(k % Ctx::kStageSlots);
        const size_t len = std::min(kStageChunk, bytes - o);
        ANQI_CUDA(c, cudaEventSynchronize(c->stage_ev[s]));  // the slot's previous copy has left it
        par_memcpy(c->stage[s], static_cast<const char*>(src) + o, len);
        ANQI_CUDA(c, cudaMemcpyAsync(static_cast<char*>(dst) + o, c->stage[s], len, cudaMemcpyHostToDevice, c->stream));
        ANQI_CUDA(c, cudaEventRecord(c->stage_ev[s], c->stream));
    }
    return ANQI_OK;
}

// Staged copies return with the data in dst; direct ones are ordered on the
// stream (the caller synchronizes before reading).
int d2h_raw(Ctx* c, void* dst, const void* src, size_t bytes) {
    if (!bytes) return ANQI_OK;
    if (!staged(c, dst, bytes)) {
        ANQI_CUDA(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
        return ANQI_OK;
    }
    const size_t nch = (bytes + kStageChunk - 1) / kStageChunk;
    auto issue = [&](size_t k) -> int {
        const int s = (int)(k % Ctx::kStageSlots);
        const size_t o = k * kStageChunk, len = std::min(kStageChunk, bytes - o);
        ANQI_CUDA(c, cudaEventSynchronize(c->stage_ev[s]));
        ANQI_CUDA(c, cudaMemcpyAsync(c->stage[s], static_cast<const char*>(src) + o, len, cudaMemcpyDeviceToHost,
                                     c->stream));
        ANQI_CUDA(c, cudaEventRecord(c->stage_ev[s], c->stream));
        return ANQI_OK;
    };
    int rc;
    for (size_t k = 0; k < nch && k < (size_t)Ctx::kStageSlots; k++)
        if ((rc = issue(k))) return rc;
    for (size_t k = 0; k < nch; k++) {
        const int s = (int)(k % Ctx::kStageSlots);
        const size_t o = k * kStageChunk, len = std::min(kStageChunk, bytes - o);
        ANQI_CUDA(c, cudaEventSynchronize(c->stage_ev[s]));
        par_memcpy(static_cast<char*>(dst) + o, c->stage[s], len);
        if (k + Ctx::kStageSlots < nch && (rc = issue(k + Ctx::kStageSlots))) return rc;
    }
    return ANQI_OK;
}

int h2d(Ctx* c, DevBuf& b, const void* src, size_t bytes) {
    int rc = ensure(c, b, bytes);
    if (rc) return rc;
    return h2d_raw(c, b.p, src, bytes);
}

int d2h(Ctx* c, void* dst, const DevBuf& b, size_t bytes) { return d2h_raw(c, dst, b.p, bytes); }

int sync(Ctx* c) {
    ANQI_CUDA(c, cudaStreamSynchronize(c->stream));
    return ANQI_OK;
}

// L2 set-aside for one hot device range accessed on the context's stream (the
// per-warp visited tables): accesses inside the window persist in L2, others
// are unaffected.  The set-aside is a limit of this process's CUDA context;
// clear_l2_window (and context teardown) returns it.
void set_l2_window(Ctx* c, const void* p, size_t bytes) {
    int maxwin = 0, maxpers = 0;
    cudaDeviceGetAttribute(&maxwin, cudaDevAttrMaxAccessPolicyWindowSize, c->device);
    cudaDeviceGetAttribute(&maxpers, cudaDevAttrMaxPersistingL2CacheSize, c->device);
    if (maxwin <= 0 || maxpers <= 0 || !p || bytes == 0) return;
    const size_t win = std::min<size_t>(bytes, (size_t)maxwin);
    const size_t keep = std::min<size_t>(win, (size_t)maxpers);
    if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, keep) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    cudaStreamAttrValue av{};
    av.accessPolicyWindow.base_ptr = const_cast<void*>(p);
    av.accessPolicyWindow.num_bytes = win;
    av.accessPolicyWindow.hitRatio = (float)keep / (float)win;
    av.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    av.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    if (cudaStreamSetAttribute(c->stream, cudaStreamAttributeAccessPolicyWindow, &av) != cudaSuccess) cudaGetLastError();
}

void clear_l2_window(Ctx* c) {
    cudaStreamAttrValue av{};
    av.accessPolicyWindow.base_ptr = nullptr;
    av.accessPolicyWindow.num_bytes = 0;
    av.accessPolicyWindow.hitRatio = 0.f;
    av.accessPolicyWindow.hitProp = cudaAccessPropertyNormal;
    av.accessPolicyWindow.missProp = cudaAccessPropertyNormal;
    if (cudaStreamSetAttribute(c->stream, cudaStreamAttributeAccessPolicyWindow, &av) != cudaSuccess) cudaGetLastError();
    if (cudaCtxResetPersistingL2Cache() != cudaSuccess) cudaGetLastError();
    if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0) != cudaSuccess) cudaGetLastError();
}

int check_device_error(Ctx* c, const char* stage) {
    uint32_t e = 0;
    ANQI_CUDA(c, cudaMemcpyAsync(&e, c->err.p, 4, cudaMemcpyDeviceToHost, c->stream));
    ANQI_CUDA(c, cudaStreamSynchronize(c->stream));
    if (e == kDevOk) return ANQI_OK;
    ANQI_CUDA(c, cudaMemsetAsync(c->err.p, 0, 4, c->stream));
    switch (e) {
        case kDevCandOverflow: return fail(c, ANQI_ERR_CAPACITY, "%s: per-query candidate capacity exceeded", stage);
        case kDevOutOverflow: return fail(c, ANQI_ERR_CAPACITY, "%s: output capacity exceeded", stage);
        case kDevPoolOverflow: return fail(c, ANQI_ERR_CAPACITY, "%s: gather pool capacity exceeded", stage);
        case kDevSortOverflow: return fail(c, ANQI_ERR_CAPACITY, "%s: sort capacity exceeded", stage);
        case kDevBadId: return fail(c, ANQI_ERR_FORMAT, "%s: an id out of range was read", stage);
        case kDevWaitTimeout: return fail(c, ANQI_ERR_TIMEOUT, "%s: a bounded device wait timed out", stage);
        default: return fail(c, ANQI_ERR_DEVICE, "%s: device error word %u", stage, e);
    }
}

__global__ void pad_rows_kernel(const float* __restrict__ src, float* __restrict__ dst, uint64_t n, uint32_t d,
                                uint32_t stride) {
    uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t total = n * stride;
    for (; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t r = t / stride;
        uint32_t j = (uint32_t)(t % stride);
        dst[t] = j < d ? src[r * d + j] : 0.0f;
    }
}

int upload_padded(Ctx* c, DevBuf& b, const float* src, uint64_t n, uint32_t d, uint32_t stride) {
    int rc = ensure(c, b, (size_t)n * stride * 4 + 64);
    if (rc) return rc;
    if (stride == d) return h2d_raw(c, b.p, src, (size_t)n * d * 4);
    TmpBuf tmp(c);
    rc = ensure(c, tmp, (size_t)n * d * 4);
    if (rc) return rc;
    if ((rc = h2d_raw(c, tmp.p, src, (size_t)n * d * 4))) return rc;
    pad_rows_kernel<<<c->sm_count * 8, 256, 0, c->stream>>>(tmp.as<float>(), b.as<float>(), n, d, stride);
    ANQI_CUDA(c, cudaGetLastError());
    ANQI_CUDA(c, cudaStreamSynchronize(c->stream));
    return ANQI_OK;
}

// IP(x, x) per row in the AVX lane order (NormSIMD16ExtAVX512__ / the
// verifier's IP(o, o)); one 4-thread group per row.
__global__ void norms_kernel(const float* __restrict__ x, uint64_t n, uint32_t dim, uint32_t stride,
                             float* __restrict__ out) {
    const uint32_t lane = threadIdx.x & 31u, gt = lane & 3u, gw = lane >> 2;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t base = warp * 8; base < n; base += nwarps * 8) {
        const uint64_t row = base + gw;
        const bool ok = row < n;
        const float* r = x + (ok ? row : base) * stride;
        float v = group_ip(r, r, dim, gt, 0xFFFFFFFFu);
        if (ok && gt == 0) out[row] = v;
    }
}

int compute_norms_device(Ctx* c, const float* d_x, uint64_t n, uint32_t dim, uint32_t stride, float* d_out) {
    const int threads = 256;
    uint64_t groups = n;
    int blocks = (int)std::min<uint64_t>((groups * 4 + threads - 1) / threads, (uint64_t)c->sm_count * 16);
    if (blocks < 1) blocks = 1;
    norms_kernel<<<blocks, threads, 0, c->stream>>>(d_x, n, dim, stride, d_out);
    ANQI_CUDA(c, cudaGetLastError());
    return ANQI_OK;
}

// G threads per pair (4, 8 or 16): the same results bit for bit.
template <int G>
__global__ void pair_dist_kernel(const float* __restrict__ a, const float* __restrict__ b, uint64_t m,
                                 uint32_t dim, uint32_t stride, float* __restrict__ l2, float* __restrict__ ip) {
    constexpr uint32_t R = 32 / G;
    const uint32_t lane = threadIdx.x & 31u, gt = lane % G, gw = lane / G;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t base = warp * R; base < m; base += nwarps * R) {
        const uint64_t row = base + gw;
        const bool ok = row < m;
        const uint64_t r = ok ? row : base;
        float v1, v2;
        if constexpr (G == 4) {
            v1 = group_l2sqr(a + r * stride, b + r * stride, dim, gt, 0xFFFFFFFFu);
            v2 = group_ip(a + r * stride, b + r * stride, dim, gt, 0xFFFFFFFFu);
        } else {
            v1 = group_l2sqr_w<G>(a + r * stride, b + r * stride, dim, gt, 0xFFFFFFFFu);
            v2 = group_ip_w<G>(a + r * stride, b + r * stride, dim, gt, 0xFFFFFFFFu);
        }
        if (ok && gt == 0) {
            l2[row] = v1;
            ip[row] = v2;
        }
    }
}

// 4 threads per pair on rows in chunk column order (common.cuh), the layout
// of the d = 128 search's lifted rows: squared L2 only.
template <uint32_t kDim>
__global__ void pair_dist_cols_kernel(const float* __restrict__ a, const float* __restrict__ b, uint64_t m,
                                      uint32_t stride, float* __restrict__ l2) {
    const uint32_t lane = threadIdx.x & 31u, gt = lane & 3u, gw = lane >> 2;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t base = warp * 8; base < m; base += nwarps * 8) {
        const uint64_t row = base + gw;
        const bool ok = row < m;
        const uint64_t r = ok ? row : base;
        const float v = group_l2sqr_cols<kDim>(a + r * stride, b + r * stride, gt, 0xFFFFFFFFu);
        if (ok && gt == 0) l2[row] = v;
    }
}

// dst row i = src row i with each full 16-float chunk in chunk column order.
__global__ void chunk_cols_kernel(const float* __restrict__ src, float* __restrict__ dst, uint64_t n,
                                  uint32_t stride, uint32_t full) {
    const uint64_t total = n * stride;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t row = e / stride;
        const uint32_t j = (uint32_t)(e - row * stride);
        dst[e] = src[row * stride + chunk_col_pos(j, full)];
    }
}

int chunk_cols(Ctx* c, const float* src, float* dst, uint64_t n, uint32_t stride, uint32_t full) {
    chunk_cols_kernel<<<c->sm_count * 8, 256, 0, c->stream>>>(src, dst, n, stride, full);
    ANQI_CUDA(c, cudaGetLastError());
    return ANQI_OK;
}

// three-phase exclusive scan: block sums, one-block scan of the sums, apply
constexpr uint32_t kScanBlock = 1024;

__global__ void scan_block_sums_kernel(const uint32_t* __restrict__ in, uint64_t n, uint64_t* __restrict__ bsum) {
    __shared__ uint64_t s[32];
    const uint64_t i = (uint64_t)blockIdx.x * kScanBlock + threadIdx.x;
    uint64_t v = i < n ? in[i] : 0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t t = 0;
        for (int w = 0; w < (int)(kScanBlock / 32); w++) t += s[w];
        bsum[blockIdx.x] = t;
    }
}

__global__ void scan_sums_kernel(uint64_t* __restrict__ bsum, uint64_t nb) {
    __shared__ uint64_t part[1024];
    const uint64_t chunk = (nb + blockDim.x - 1) / blockDim.x;
    const uint64_t b = min(nb, threadIdx.x * chunk), e = min(nb, b + chunk);
    uint64_t s = 0;
    for (uint64_t i = b; i < e; i++) s += bsum[i];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t run = 0;
        for (uint32_t i = 0; i < blockDim.x; i++) {
            const uint64_t v = part[i];
            part[i] = run;
            run += v;
        }
    }
    __syncthreads();
    uint64_t run = part[threadIdx.x];
    for (uint64_t i = b; i < e; i++) {
        const uint64_t v = bsum[i];
        bsum[i] = run;
        run += v;
    }
}

__global__ void scan_apply_kernel(const uint32_t* __restrict__ in, uint64_t n, const uint64_t* __restrict__ bsum,
                                  uint64_t* __restrict__ out) {
    __shared__ uint64_t s[32];
    const uint64_t i = (uint64_t)blockIdx.x * kScanBlock + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint64_t v = i < n ? in[i] : 0;
    uint64_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) s[w] = x;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint64_t y = threadIdx.x < kScanBlock / 32 ? s[threadIdx.x] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t z = __shfl_up_sync(0xFFFFFFFFu, y, o);
            if (threadIdx.x >= (uint32_t)o) y += z;
        }
        s[threadIdx.x] = y;
    }
    __syncthreads();
    const uint64_t before = (w ? s[w - 1] : 0) + x - v + bsum[blockIdx.x];
    if (i < n) out[i] = before;
    if (i == n - 1) out[n] = before + v;
}

int device_scan(Ctx* c, const uint32_t* d_in, uint64_t* d_out, uint64_t n) {
    if (n == 0) {
        ANQI_CUDA(c, cudaMemsetAsync(d_out, 0, 8, c->stream));
        return ANQI_OK;
    }
    const uint64_t nb = (n + kScanBlock - 1) / kScanBlock;
    TmpBuf bs(c);
    int rc = ensure(c, bs, nb * 8);
    if (rc) return rc;
    scan_block_sums_kernel<<<(unsigned)nb, kScanBlock, 0, c->stream>>>(d_in, n, bs.as<uint64_t>());
    scan_sums_kernel<<<1, 1024, 0, c->stream>>>(bs.as<uint64_t>(), nb);
    scan_apply_kernel<<<(unsigned)nb, kScanBlock, 0, c->stream>>>(d_in, n, bs.as<uint64_t>(), d_out);
    ANQI_CUDA(c, cudaGetLastError());
    return sync(c);
}

}  // namespace anqi

using namespace anqi;

extern "C" {

int anqi_version(void) { return 1; }

int anqi_inject_fault(anqi_ctx* h, uint32_t flags) {
    if (!h || (flags & ~ANQI_FAULT_DROP_ROW_COPIES)) return ANQI_ERR_ARGS;
    h->c.inject = flags;
    return ANQI_OK;
}

int anqi_ctx_create(int device, anqi_ctx** out) {
    if (!out) return ANQI_ERR_ARGS;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return ANQI_ERR_DEVICE;
    if (device < 0 || device >= count) return ANQI_ERR_ARGS;
    if (cudaSetDevice(device) != cudaSuccess) return ANQI_ERR_DEVICE;
    anqi_ctx* h = new anqi_ctx();
    Ctx* c = &h->c;
    c->device = device;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        delete h;
        return ANQI_ERR_DEVICE;
    }
    c->sm_count = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
        cudaEventCreate(&c->ev2) != cudaSuccess || cudaEventCreate(&c->ev3) != cudaSuccess) {
        delete h;
        return ANQI_ERR_DEVICE;
    }
    if (ensure(c, c->err, 64) || ensure(c, c->counters, 4096)) {
        delete h;
        return ANQI_ERR_DEVICE;
    }
    cudaMemsetAsync(c->err.p, 0, 64, c->stream);
    cudaStreamSynchronize(c->stream);
    *out = h;
    return ANQI_OK;
}

void anqi_ctx_destroy(anqi_ctx* h) {
    if (!h) return;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->l2_window) clear_l2_window(c);
    if (c->qgraph) cudaGraphExecDestroy(c->qgraph);
    for (DevBuf* b : c->member_bufs()) release(c, *b);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->ev2) cudaEventDestroy(c->ev2);
    if (c->ev3) cudaEventDestroy(c->ev3);
    if (c->tev0) cudaEventDestroy(c->tev0);
    if (c->tev1) cudaEventDestroy(c->tev1);
    for (int s = 0; s < Ctx::kStageSlots; s++) {
        if (c->stage[s]) cudaFreeHost(c->stage[s]);
        if (c->stage_ev[s]) cudaEventDestroy(c->stage_ev[s]);
    }
    if (c->stream) cudaStreamDestroy(c->stream);
    delete h;
}

const char* anqi_last_error(const anqi_ctx* h) { return h ? h->c.last_error.c_str() : "null context"; }

uint64_t anqi_device_bytes(const anqi_ctx* h) { return h ? h->c.device_bytes : 0; }

int anqi_timer_start(anqi_ctx* h) {
    if (!h) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    if (!c->tev0) {
        ANQI_CUDA(c, cudaEventCreate(&c->tev0));
        ANQI_CUDA(c, cudaEventCreate(&c->tev1));
    }
    ANQI_CUDA(c, cudaEventRecord(c->tev0, c->stream));
    return ANQI_OK;
}

int anqi_timer_stop(anqi_ctx* h, float* ms) {
    if (!h || !ms) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    if (!c->tev0) return fail(c, ANQI_ERR_ARGS, "anqi_timer_stop without anqi_timer_start");
    ANQI_CUDA(c, cudaEventRecord(c->tev1, c->stream));
    ANQI_CUDA(c, cudaEventSynchronize(c->tev1));
    ANQI_CUDA(c, cudaEventElapsedTime(ms, c->tev0, c->tev1));
    return ANQI_OK;
}

int anqi_pair_distances(anqi_ctx* h, const float* a, const float* b, uint64_t m, uint32_t dim, float* l2sqr,
                        float* ip) {
    return anqi_pair_distances_group(h, a, b, m, dim, 4, l2sqr, ip);
}

int anqi_pair_distances_group(anqi_ctx* h, const float* a, const float* b, uint64_t m, uint32_t dim,
                              uint32_t group, float* l2sqr, float* ip) {
    if (!h || !a || !b || !l2sqr || !ip || dim == 0 || (group != 0 && group != 4 && group != 8 && group != 16) ||
        (group == 0 && dim != 130))
        return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    if (m == 0) return ANQI_OK;
    const uint32_t stride = round_up(dim, 8);
    TmpBuf da(c), db(c), dl(c), di(c);
    int rc;
    if ((rc = upload_padded(c, da, a, m, dim, stride)) || (rc = upload_padded(c, db, b, m, dim, stride)) ||
        (rc = ensure(c, dl, m * 4)) || (rc = ensure(c, di, m * 4)))
        return rc;
    int blocks = (int)std::min<uint64_t>((m * 4 + 255) / 256, (uint64_t)c->sm_count * 16);
    if (group == 0) {
        // ip through the 4-thread form, then l2 (overwritten) through the
        // chunk-column one
        TmpBuf ca(c), cb(c);
        if ((rc = ensure(c, ca, m * (size_t)stride * 4)) || (rc = ensure(c, cb, m * (size_t)stride * 4))) return rc;
        pair_dist_kernel<4><<<blocks, 256, 0, c->stream>>>(da.as<float>(), db.as<float>(), m, dim, stride,
                                                           dl.as<float>(), di.as<float>());
        chunk_cols_kernel<<<c->sm_count * 8, 256, 0, c->stream>>>(da.as<float>(), ca.as<float>(), m, stride, 128);
        chunk_cols_kernel<<<c->sm_count * 8, 256, 0, c->stream>>>(db.as<float>(), cb.as<float>(), m, stride, 128);
        pair_dist_cols_kernel<130><<<blocks, 256, 0, c->stream>>>(ca.as<float>(), cb.as<float>(), m, stride,
                                                                  dl.as<float>());
        ANQI_CUDA(c, cudaGetLastError());
        if ((rc = d2h(c, l2sqr, dl, m * 4)) || (rc = d2h(c, ip, di, m * 4)) || (rc = sync(c))) return rc;
        return ANQI_OK;
    }
    auto kern = group == 4 ? pair_dist_kernel<4> : group == 8 ? pair_dist_kernel<8> : pair_dist_kernel<16>;
    kern<<<blocks, 256, 0, c->stream>>>(da.as<float>(), db.as<float>(), m, dim, stride, dl.as<float>(),
                                        di.as<float>());
    ANQI_CUDA(c, cudaGetLastError());
    if ((rc = d2h(c, l2sqr, dl, m * 4)) || (rc = d2h(c, ip, di, m * 4)) || (rc = sync(c))) return rc;
    return ANQI_OK;
}

}  // extern "C"
