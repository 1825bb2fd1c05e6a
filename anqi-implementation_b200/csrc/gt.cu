// Exact reverse-kNN membership (the evaluation ground truth).
//
// Reference: tools/dataset_gt.cpp:270-313 (--mode ground-truth): for every
// query q, all base rows j with key = |q|^2 + |b_j|^2 - 2 <q, b_j> <= rk2[j],
// sorted by (key, id); FP32 in the AVX lane order, so the CSR is bit-exact.
// The ip metric's key is -<q, b_j> (dataset_gt.cpp:288).
// Two passes over the same tiles: count hits per query, then write them at
// scanned offsets and sort each query's segment.
#include <algorithm>

#include "internal.h"
#include "util.cuh"

namespace anqi {

constexpr uint32_t kGtQ = 16;     // queries per CTA
constexpr uint32_t kGtTile = 64;  // base rows per tile (fewer for long rows, to fit shared memory)

__global__ void __launch_bounds__(256) rknn_gt_kernel(const float* __restrict__ base, const float* __restrict__ bn,
                                                      uint64_t n, const float* __restrict__ q, uint64_t nq,
                                                      uint32_t stride, uint32_t d, const float* __restrict__ rk2,
                                                      uint32_t* __restrict__ cnt, const uint64_t* __restrict__ off,
                                                      uint32_t* __restrict__ fill, uint32_t* __restrict__ out_id,
                                                      float* __restrict__ out_key, uint32_t is_ip, uint32_t tile) {
    extern __shared__ __align__(16) unsigned char sm[];
    float* qv = reinterpret_cast<float*>(sm);            // kGtQ x stride
    float* tv = qv + (size_t)kGtQ * stride;              // tile x stride
    float* qn = tv + (size_t)tile * stride;              // kGtQ
    const uint64_t q0 = (uint64_t)blockIdx.x * kGtQ;
    const uint32_t nqb = (uint32_t)min_u64(kGtQ, nq - q0);
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5, gt = lane & 3u, gw = lane >> 2;
    const uint32_t nwarp = blockDim.x >> 5;
    for (uint32_t t = threadIdx.x; t < nqb * stride; t += blockDim.x) qv[t] = q[q0 * stride + t];
    __syncthreads();
    for (uint32_t r = wib; r < nqb; r += nwarp) {
        const float v = group_ip(qv + (size_t)r * stride, qv + (size_t)r * stride, d, gt, kAll);
        if (lane == 0) qn[r] = v;
    }
    __syncthreads();
    for (uint64_t c0 = 0; c0 < n; c0 += tile) {
        const uint32_t tr = (uint32_t)min_u64(tile, n - c0);
        for (uint32_t t = threadIdx.x; t < tr * (stride / 4); t += blockDim.x)
            reinterpret_cast<float4*>(tv)[t] = reinterpret_cast<const float4*>(base + c0 * stride)[t];
        __syncthreads();
        for (uint32_t r = wib; r < nqb; r += nwarp) {
            const uint64_t qi = q0 + r;
            uint32_t local = 0;
            for (uint32_t b0 = 0; b0 < tr; b0 += 8) {
                const uint32_t j = b0 + gw;
                const bool ok = j < tr;
                const uint32_t jj = ok ? j : b0;
                const float ip = group_ip(qv + (size_t)r * stride, tv + (size_t)jj * stride, d, gt, kAll);
                const float key = is_ip ? -ip : __fsub_rn(__fadd_rn(qn[r], bn[c0 + jj]), __fmul_rn(2.0f, ip));
                const bool hit = ok && gt == 0 && key <= rk2[c0 + jj];
                if (hit) {
                    if (off) {
                        const uint32_t pos = atomicAdd(fill + qi, 1u);
                        out_id[off[qi] + pos] = (uint32_t)(c0 + jj);
                        out_key[off[qi] + pos] = key;
                    } else {
                        local++;
                    }
                }
            }
            if (!off) {
                for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(kAll, local, o);
                if (lane == 0 && local) cnt[qi] += local;
            }
        }
        __syncthreads();
    }
}

__global__ void sort_segments_kernel(const uint64_t* __restrict__ off, uint64_t nq, uint32_t* __restrict__ ids,
                                     float* __restrict__ keys, float* __restrict__ scr_d, uint32_t* __restrict__ scr_i,
                                     uint32_t scr_cap) {
    extern __shared__ __align__(16) unsigned char sm[];
    constexpr uint32_t kSm = 1024;
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    float* sd = reinterpret_cast<float*>(sm) + wib * 2 * kSm;
    uint32_t* si = reinterpret_cast<uint32_t*>(sd + kSm);
    const uint32_t slot = blockIdx.x * (blockDim.x >> 5) + wib;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const float inf = __int_as_float(0x7f800000);
    for (uint64_t qi = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; qi < nq; qi += nw) {
        const uint64_t o = off[qi];
        const uint32_t m = (uint32_t)(off[qi + 1] - o);
        if (m < 2) continue;
        const uint32_t np2 = next_pow2(m);
        float* bd = np2 <= kSm ? sd : scr_d + (size_t)slot * scr_cap;
        uint32_t* bi = np2 <= kSm ? si : scr_i + (size_t)slot * scr_cap;
        for (uint32_t t = lane; t < np2; t += 32) {
            bd[t] = t < m ? keys[o + t] : inf;
            bi[t] = t < m ? ids[o + t] : kEmpty;
        }
        __syncwarp();
        warp_sort_pairs(bd, bi, np2);
        for (uint32_t t = lane; t < m; t += 32) {
            keys[o + t] = bd[t];
            ids[o + t] = bi[t];
        }
        __syncwarp();
    }
}

// Sorts every CSR segment [off[i], off[i+1]) of (keys, ids) by (key, id).
int sort_csr_segments(Ctx* c, const uint64_t* d_off, uint64_t nseg, uint32_t* d_ids, float* d_keys, uint64_t maxm) {
    const uint32_t scr_cap = maxm > 1024 ? (uint32_t)(1ull << (64 - __builtin_clzll(maxm - 1))) : 1;
    const uint32_t sblocks = (uint32_t)c->sm_count * 4;
    TmpBuf sd(c), si(c);
    int rc;
    if ((rc = ensure(c, sd, (size_t)sblocks * 4 * scr_cap * 4)) || (rc = ensure(c, si, (size_t)sblocks * 4 * scr_cap * 4)))
        return rc;
    const size_t ssm = 4 * 2 * 1024 * 4;
    ANQI_CUDA(c, cudaFuncSetAttribute(sort_segments_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssm));
    sort_segments_kernel<<<sblocks, 128, ssm, c->stream>>>(d_off, nseg, d_ids, d_keys, sd.as<float>(),
                                                           si.as<uint32_t>(), scr_cap);
    ANQI_CUDA(c, cudaGetLastError());
    return sync(c);
}

}  // namespace anqi

using namespace anqi;

extern "C" int anqi_rknn_ground_truth(anqi_ctx* h, const float* base, uint64_t n, const float* query, uint64_t nq,
                                      uint32_t d, const float* rk2, uint32_t* off, uint32_t* ids, float* keys,
                                      uint64_t cap, uint64_t* total) {
    return anqi_rknn_ground_truth_metric(h, base, n, query, nq, d, rk2, ANQI_METRIC_L2, off, ids, keys, cap, total);
}

extern "C" int anqi_rknn_ground_truth_metric(anqi_ctx* h, const float* base, uint64_t n, const float* query,
                                             uint64_t nq, uint32_t d, const float* rk2, uint32_t metric, uint32_t* off,
                                             uint32_t* ids, float* keys, uint64_t cap, uint64_t* total) {
    if (!h || !base || !query || !rk2 || !off || n == 0 || nq == 0 || d == 0 || metric > ANQI_METRIC_IP)
        return ANQI_ERR_ARGS;
    const uint32_t is_ip = metric == ANQI_METRIC_IP;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    const uint32_t xs = round_up(d, 8);
    TmpBuf db(c), dq(c), dbn(c), dr(c), dcnt(c), doff(c), dfill(c), did(c), dkey(c);
    int rc;
    if ((rc = upload_padded(c, db, base, n, d, xs)) || (rc = upload_padded(c, dq, query, nq, d, xs)) ||
        (rc = ensure(c, dbn, n * 4)) || (rc = h2d(c, dr, rk2, n * 4)) || (rc = ensure(c, dcnt, nq * 4)) ||
        (rc = ensure(c, doff, (nq + 1) * 8)) || (rc = ensure(c, dfill, nq * 4)))
        return rc;
    if ((rc = compute_norms_device(c, db.as<float>(), n, d, xs, dbn.as<float>()))) return rc;
    ANQI_CUDA(c, cudaMemsetAsync(dcnt.p, 0, nq * 4, c->stream));
    ANQI_CUDA(c, cudaMemsetAsync(dfill.p, 0, nq * 4, c->stream));
    // base rows per tile: 64, or fewer (a multiple of 8) when rows are long
    uint32_t tile = kGtTile;
    while (tile > 8 && ((size_t)(kGtQ + tile) * xs + kGtQ) * 4 > 227 * 1024) tile -= 8;
    const size_t smem = ((size_t)(kGtQ + tile) * xs + kGtQ) * 4;
    if (smem > 227 * 1024) return fail(c, ANQI_ERR_ARGS, "dimension %u too large for the ground-truth kernel", d);
    ANQI_CUDA(c, cudaFuncSetAttribute(rknn_gt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const unsigned blocks = (unsigned)((nq + kGtQ - 1) / kGtQ);
    rknn_gt_kernel<<<blocks, 256, smem, c->stream>>>(db.as<float>(), dbn.as<float>(), n, dq.as<float>(), nq, xs, d,
                                                     dr.as<float>(), dcnt.as<uint32_t>(), nullptr, nullptr, nullptr,
                                                     nullptr, is_ip, tile);
    ANQI_CUDA(c, cudaGetLastError());
    if ((rc = device_scan(c, dcnt.as<uint32_t>(), doff.as<uint64_t>(), nq))) return rc;
    std::vector<uint64_t> hoff(nq + 1);
    ANQI_CUDA(c, cudaMemcpy(hoff.data(), doff.p, (nq + 1) * 8, cudaMemcpyDeviceToHost));
    const uint64_t tot = hoff[nq];
    if (total) *total = tot;
    if (tot > cap || tot > 0xFFFFFFFFull)
        return fail(c, ANQI_ERR_CAPACITY, "reverse-kNN output needs %llu entries", (unsigned long long)tot);
    if ((rc = ensure(c, did, tot * 4 + 4)) || (rc = ensure(c, dkey, tot * 4 + 4))) return rc;
    rknn_gt_kernel<<<blocks, 256, smem, c->stream>>>(db.as<float>(), dbn.as<float>(), n, dq.as<float>(), nq, xs, d,
                                                     dr.as<float>(), nullptr, doff.as<uint64_t>(), dfill.as<uint32_t>(),
                                                     did.as<uint32_t>(), dkey.as<float>(), is_ip, tile);
    ANQI_CUDA(c, cudaGetLastError());
    uint64_t maxm = 0;
    for (uint64_t i = 0; i < nq; i++) maxm = std::max(maxm, hoff[i + 1] - hoff[i]);
    const uint32_t scr_cap = maxm > 1024 ? (uint32_t)(1ull << (64 - __builtin_clzll(maxm - 1))) : 1;
    const uint32_t sblocks = (uint32_t)c->sm_count * 4;
    TmpBuf sd(c), si(c);
    if ((rc = ensure(c, sd, (size_t)sblocks * 4 * scr_cap * 4)) || (rc = ensure(c, si, (size_t)sblocks * 4 * scr_cap * 4)))
        return rc;
    const size_t ssm = 4 * 2 * 1024 * 4;
    ANQI_CUDA(c, cudaFuncSetAttribute(sort_segments_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssm));
    sort_segments_kernel<<<sblocks, 128, ssm, c->stream>>>(doff.as<uint64_t>(), nq, did.as<uint32_t>(),
                                                           dkey.as<float>(), sd.as<float>(), si.as<uint32_t>(), scr_cap);
    ANQI_CUDA(c, cudaGetLastError());
    for (uint64_t i = 0; i <= nq; i++) off[i] = (uint32_t)hoff[i];
    if (tot) {
        if (ids && (rc = d2h(c, ids, did, tot * 4))) return rc;
        if (keys && (rc = d2h(c, keys, dkey, tot * 4))) return rc;
    }
    return sync(c);
}
