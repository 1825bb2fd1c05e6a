// The d+2 lift that turns "q inside o's r_K ball" into one global range test.
//
// Reference: src/rknn_query.cpp:2203-2235 (anyk_lift, graph radius = the
// AKNN rank-K cutoff of each object; L2, or the ip metric's s^2 r coordinate).  All arithmetic is double with explicit
// _rn operations (no contraction), matching the reference compiled with
// -std=c++17.  The sum of squared norms is accumulated per row, then over rows
// in index order -- the order of the reference's OpenMP reduction at one
// thread -- so the scale s is reproducible bit for bit.
#include <algorithm>

#include "common.cuh"
#include "internal.h"

namespace anqi {

__global__ void lift_rowsum_kernel(const float* __restrict__ base, uint64_t n, uint32_t d, double* __restrict__ rs) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const float* o = base + i * d;
        double s = 0;
        for (uint32_t j = 0; j < d; j++) s = __dadd_rn(s, __dmul_rn((double)o[j], (double)o[j]));
        rs[i] = s;
    }
}

// Sequential in row order on one thread (about 1M dependent adds, a few ms).
__global__ void lift_scale_kernel(const double* __restrict__ rs, uint64_t n, double* __restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double sum = 0;
    for (uint64_t i = 0; i < n; i++) sum = __dadd_rn(sum, rs[i]);
    const double s = __ddiv_rn(1.0, __dsqrt_rn(__dadd_rn(__ddiv_rn(sum, (double)n), 1e-12)));
    out[0] = s;
    out[1] = __dmul_rn(s, s);
    out[2] = 0.0;  // running max of |h|^2 (as bits via atomicMax below)
}

__global__ void lift_rows_kernel(const float* __restrict__ base, uint64_t n, uint32_t d, const float* __restrict__ radius,
                                 const double* __restrict__ sc, float* __restrict__ lifted,
                                 unsigned long long* __restrict__ maxbits, uint32_t ip) {
    const double s = sc[0], sc2 = sc[1];
    const uint32_t dout = d + 2;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const float* o = base + i * d;
        float* h = lifted + i * dout;
        double nr2 = 0;
        for (uint32_t j = 0; j < d; j++) {
            const double v = __dmul_rn((double)o[j], s);
            h[j] = __double2float_rn(v);
            nr2 = __dadd_rn(nr2, __dmul_rn(v, v));
        }
        // the ip metric's coordinate is s^2 r (rknn_query.cpp:2227)
        const float hd = ip ? __double2float_rn(__dmul_rn((double)radius[i], sc2))
                            : __double2float_rn(__dmul_rn(0.5, __dsub_rn(__dmul_rn((double)radius[i], sc2), nr2)));
        h[d] = hd;
        const double hn2 = __dadd_rn(nr2, __dmul_rn((double)hd, (double)hd));
        atomicMax(maxbits, (unsigned long long)__double_as_longlong(hn2));
    }
}

__global__ void lift_pad_kernel(uint64_t n, uint32_t d, const unsigned long long* __restrict__ maxbits,
                                float* __restrict__ lifted, double* __restrict__ m2out) {
    const double M2 = __dmul_rn(__longlong_as_double((long long)*maxbits), 1.0001);
    if (blockIdx.x == 0 && threadIdx.x == 0) *m2out = M2;
    const uint32_t dl = d + 1, dout = d + 2;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        float* h = lifted + i * dout;
        double hn2 = 0;
        for (uint32_t j = 0; j < dl; j++) hn2 = __dadd_rn(hn2, __dmul_rn((double)h[j], (double)h[j]));
        double pad = __dsub_rn(M2, hn2);
        if (pad < 0) pad = 0;
        h[dl] = __double2float_rn(__dsqrt_rn(pad));
    }
}

}  // namespace anqi

using namespace anqi;

extern "C" {

int anqi_lift(anqi_ctx* h, const float* base, uint64_t n, uint32_t d, const float* radius, float* lifted,
              double* mstar2, double* scale) {
    return anqi_lift_metric(h, base, n, d, radius, ANQI_METRIC_L2, lifted, mstar2, scale);
}

int anqi_lift_metric(anqi_ctx* h, const float* base, uint64_t n, uint32_t d, const float* radius, uint32_t metric,
                     float* lifted, double* mstar2, double* scale) {
    if (!h || !base || !radius || !lifted || !mstar2 || !scale || n == 0 || d == 0 || metric > ANQI_METRIC_IP)
        return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    TmpBuf db(c), dr(c), drs(c), dsc(c), dl(c), dmax(c);
    int rc;
    if ((rc = h2d(c, db, base, n * d * 4)) || (rc = h2d(c, dr, radius, n * 4)) || (rc = ensure(c, drs, n * 8)) ||
        (rc = ensure(c, dsc, 64)) || (rc = ensure(c, dl, n * (d + 2ull) * 4)) || (rc = ensure(c, dmax, 16)))
        return rc;
    ANQI_CUDA(c, cudaMemsetAsync(dmax.p, 0, 16, c->stream));
    const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)c->sm_count * 8));
    lift_rowsum_kernel<<<blocks, 256, 0, c->stream>>>(db.as<float>(), n, d, drs.as<double>());
    lift_scale_kernel<<<1, 32, 0, c->stream>>>(drs.as<double>(), n, dsc.as<double>());
    lift_rows_kernel<<<blocks, 256, 0, c->stream>>>(db.as<float>(), n, d, dr.as<float>(), dsc.as<double>(),
                                                   dl.as<float>(), dmax.as<unsigned long long>(),
                                                   metric == ANQI_METRIC_IP);
    lift_pad_kernel<<<blocks, 256, 0, c->stream>>>(n, d, dmax.as<unsigned long long>(), dl.as<float>(),
                                                  dsc.as<double>() + 3);
    ANQI_CUDA(c, cudaGetLastError());
    double sc[4];
    if ((rc = d2h(c, lifted, dl, n * (d + 2ull) * 4))) return rc;
    ANQI_CUDA(c, cudaMemcpyAsync(sc, dsc.p, 32, cudaMemcpyDeviceToHost, c->stream));
    if ((rc = sync(c))) return rc;
    *scale = sc[0];
    *mstar2 = sc[3];
    return ANQI_OK;
}

}  // extern "C"
