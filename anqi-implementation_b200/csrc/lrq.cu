// Rank-M + packed-u8 LRQ verifier codec (floor policy).
//
// Reference: CompactLrqVerifier::build / materialize_k, src/rknn_query.cpp:679-753,
// with encode_learned_residual (rknn_query.cpp:482-513) and the packed-code
// accessors of include/packed_code_array.h:18-63 (u8: one byte per code).
//
// The reference evaluates every sum in double without fused multiply-adds
// (-std=c++17 turns contraction off); every operation here is an explicit _rn
// intrinsic so nvcc cannot fuse them either.  On the device the codes are kept
// k-major (nk rows of n4 = round_up(n, 4) bytes) so materializing one rank reads
// a contiguous byte column; four codes arrive in one 32-bit load and are split
// with __byte_perm.
#include <algorithm>

#include "common.cuh"
#include "internal.h"

namespace anqi {

constexpr int kEncodeRows = 32;  // rows staged per block

// One thread per row; keys for kEncodeRows rows staged in shared memory.
__global__ void lrq_encode_kernel(const float* __restrict__ keys, uint64_t n, uint32_t nk, uint32_t rankm,
                                  const float* __restrict__ mu, const float* __restrict__ basis,
                                  const float* __restrict__ codebook, uint32_t code_size,
                                  float* __restrict__ coeff, uint8_t* __restrict__ codes) {
    extern __shared__ float sh[];
    float* s_keys = sh;                                  // kEncodeRows x nk
    float* s_mu = s_keys + (size_t)kEncodeRows * nk;     // nk
    float* s_basis = s_mu + nk;                          // rankm x nk
    const uint64_t row0 = (uint64_t)blockIdx.x * kEncodeRows;
    const uint32_t rows = (uint32_t)((n - row0) < (uint64_t)kEncodeRows ? (n - row0) : (uint64_t)kEncodeRows);
    for (uint32_t t = threadIdx.x; t < rows * nk; t += blockDim.x) s_keys[t] = keys[row0 * nk + t];
    for (uint32_t t = threadIdx.x; t < nk; t += blockDim.x) s_mu[t] = mu[t];
    for (uint32_t t = threadIdx.x; t < rankm * nk; t += blockDim.x) s_basis[t] = basis[t];
    __syncthreads();
    const uint32_t r = threadIdx.x;
    if (r < rows) {
        const float* rk = s_keys + (size_t)r * nk;
        float ci[16];
        for (uint32_t m = 0; m < rankm; m++) {
            double c = 0.0;
            for (uint32_t k = 0; k < nk; k++)
                c = __dadd_rn(c, __dmul_rn(__dsub_rn((double)rk[k], (double)s_mu[k]), (double)s_basis[m * nk + k]));
            ci[m] = __double2float_rn(c);
            coeff[(row0 + r) * rankm + m] = ci[m];
        }
        for (uint32_t k = 0; k < nk; k++) {
            double recon = (double)s_mu[k];
            for (uint32_t m = 0; m < rankm; m++)
                recon = __dadd_rn(recon, __dmul_rn((double)ci[m], (double)s_basis[m * nk + k]));
            const float v = __double2float_rn(__dsub_rn((double)rk[k], recon));
            // floor: last centre <= v (upper_bound - 1), clamped to 0
            const float* c = codebook + (size_t)k * code_size;
            uint32_t lo = 0, hi = code_size;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (v < __ldg(c + mid)) hi = mid;
                else lo = mid + 1;
            }
            s_keys[(size_t)r * nk + k] = __uint_as_float(lo == 0 ? 0u : lo - 1);
        }
    }
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < rows * nk; t += blockDim.x)
        codes[row0 * nk + t] = (uint8_t)__float_as_uint(s_keys[t]);
}

// Object-major codes (n x nk) -> k-major (nk x n4), 32 x 32 tiles.
__global__ void codes_transpose_kernel(const uint8_t* __restrict__ src, uint64_t n, uint32_t nk, uint64_t n4,
                                       uint8_t* __restrict__ dst) {
    __shared__ uint8_t tile[32][33];
    const uint64_t o0 = (uint64_t)blockIdx.x * 32;
    const uint32_t k0 = blockIdx.y * 32;
    for (uint32_t y = threadIdx.y; y < 32; y += blockDim.y) {
        const uint64_t o = o0 + y;
        const uint32_t k = k0 + threadIdx.x;
        tile[y][threadIdx.x] = (o < n && k < nk) ? src[o * nk + k] : 0;
    }
    __syncthreads();
    for (uint32_t y = threadIdx.y; y < 32; y += blockDim.y) {
        const uint32_t k = k0 + y;
        const uint64_t o = o0 + threadIdx.x;
        if (k < nk && o < n4) dst[(uint64_t)k * n4 + o] = tile[threadIdx.x][y];
    }
}

// thr[o] = f32(max(0, scale * (mu_k + sum_m c_om G_mk + cb_k[code]))), four objects per thread.
__global__ void lrq_materialize_kernel(const float* __restrict__ coeff, const uint8_t* __restrict__ codes_t,
                                       uint64_t n, uint64_t n4, uint32_t nk, uint32_t rankm,
                                       const float* __restrict__ mu, const float* __restrict__ basis,
                                       const float* __restrict__ codebook, uint32_t code_size, uint32_t k,
                                       double radius_scale, float* __restrict__ thr) {
    __shared__ double s_g[16];
    if (threadIdx.x < rankm) s_g[threadIdx.x] = (double)basis[threadIdx.x * nk + k];
    __syncthreads();
    const double muk = (double)mu[k];
    const float* cb = codebook + (size_t)k * code_size;
    const uint8_t* col = codes_t + (uint64_t)k * n4;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; 4 * t < n;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t word = *reinterpret_cast<const uint32_t*>(col + 4 * t);
#pragma unroll
        for (uint32_t j = 0; j < 4; j++) {
            const uint64_t o = 4 * t + j;
            if (o >= n) break;
            const uint32_t code = __byte_perm(word, 0u, 0x4440u | j);
            const float* ci = coeff + o * rankm;
            double value = muk;
            for (uint32_t m = 0; m < rankm; m++) value = __dadd_rn(value, __dmul_rn((double)ci[m], s_g[m]));
            value = __dadd_rn(value, (double)__ldg(cb + code));
            const double scaled = __dmul_rn(radius_scale, value);
            thr[o] = __double2float_rn(0.0 < scaled ? scaled : 0.0);
        }
    }
}

int lrq_materialize_device(Ctx* c, const Verifier& v, uint32_t k, double scale, float* d_out) {
    const uint64_t n4 = (v.n + 3) / 4 * 4;
    int blocks = (int)std::min<uint64_t>((v.n / 4 + 256) / 256, (uint64_t)c->sm_count * 8);
    lrq_materialize_kernel<<<std::max(blocks, 1), 256, 0, c->stream>>>(
        v.coeff.as<float>(), v.codes_t.as<uint8_t>(), v.n, n4, v.nk, v.rankm, v.mu.as<float>(), v.basis.as<float>(),
        v.codebook.as<float>(), v.code_size, k - 1, scale, d_out);
    ANQI_CUDA(c, cudaGetLastError());
    return ANQI_OK;
}

static int check_lrq_args(Ctx* c, uint64_t n, uint32_t nk, uint32_t rankm, const float* codebook, uint32_t code_size) {
    if (n == 0 || nk == 0 || rankm == 0 || rankm > 16 || code_size != 256)
        return fail(c, ANQI_ERR_ARGS, "invalid CompactLrqVerifier configuration (n=%llu nk=%u rankm=%u code_size=%u)",
                    (unsigned long long)n, nk, rankm, code_size);
    for (uint32_t k = 0; k < nk; k++)
        for (uint32_t j = 1; j < code_size; j++)
            if (codebook[(size_t)k * code_size + j] < codebook[(size_t)k * code_size + j - 1])
                return fail(c, ANQI_ERR_FORMAT, "LRQ codebook row is not sorted: k=%u", k + 1);
    return ANQI_OK;
}

static int load_verifier(Ctx* c, Verifier& v, const float* coeff, const uint8_t* codes, uint64_t n, uint32_t nk,
                         uint32_t rankm, const float* mu, const float* basis, const float* codebook,
                         uint32_t code_size) {
    int rc = check_lrq_args(c, n, nk, rankm, codebook, code_size);
    if (rc) return rc;
    v.loaded = false;
    v.n = n;
    v.nk = nk;
    v.rankm = rankm;
    v.code_size = code_size;
    const uint64_t n4 = (n + 3) / 4 * 4;
    TmpBuf raw(c);
    if ((rc = h2d(c, v.coeff, coeff, n * rankm * 4)) || (rc = h2d(c, raw, codes, n * nk)) ||
        (rc = ensure(c, v.codes_t, nk * n4)) || (rc = h2d(c, v.mu, mu, nk * 4)) ||
        (rc = h2d(c, v.basis, basis, (size_t)rankm * nk * 4)) ||
        (rc = h2d(c, v.codebook, codebook, (size_t)nk * code_size * 4)))
        return rc;
    dim3 grid((unsigned)((n4 + 31) / 32), (nk + 31) / 32), block(32, 8);
    codes_transpose_kernel<<<grid, block, 0, c->stream>>>(raw.as<uint8_t>(), n, nk, n4, v.codes_t.as<uint8_t>());
    ANQI_CUDA(c, cudaGetLastError());
    if ((rc = sync(c))) return rc;
    v.loaded = true;
    return ANQI_OK;
}

}  // namespace anqi

using namespace anqi;

extern "C" {

int anqi_lrq_encode(anqi_ctx* h, const float* keys, uint64_t n, uint32_t nk, uint32_t rankm, const float* mu,
                    const float* basis, const float* codebook, uint32_t code_size, float* coeff, uint8_t* codes) {
    if (!h || !keys || !mu || !basis || !codebook || !coeff || !codes) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    int rc = check_lrq_args(c, n, nk, rankm, codebook, code_size);
    if (rc) return rc;
    TmpBuf dk(c), dmu(c), db(c), dcb(c), dco(c), dcd(c);
    if ((rc = h2d(c, dk, keys, n * nk * 4)) || (rc = h2d(c, dmu, mu, nk * 4)) ||
        (rc = h2d(c, db, basis, (size_t)rankm * nk * 4)) || (rc = h2d(c, dcb, codebook, (size_t)nk * code_size * 4)) ||
        (rc = ensure(c, dco, n * rankm * 4)) || (rc = ensure(c, dcd, n * nk)))
        return rc;
    const size_t smem = ((size_t)kEncodeRows * nk + nk + (size_t)rankm * nk) * 4;
    if (smem > 200 * 1024) return fail(c, ANQI_ERR_ARGS, "nk too large for the encoder");
    ANQI_CUDA(c, cudaFuncSetAttribute(lrq_encode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const unsigned blocks = (unsigned)((n + kEncodeRows - 1) / kEncodeRows);
    lrq_encode_kernel<<<blocks, kEncodeRows, smem, c->stream>>>(dk.as<float>(), n, nk, rankm, dmu.as<float>(),
                                                                db.as<float>(), dcb.as<float>(), code_size,
                                                                dco.as<float>(), dcd.as<uint8_t>());
    ANQI_CUDA(c, cudaGetLastError());
    if ((rc = d2h(c, coeff, dco, n * rankm * 4)) || (rc = d2h(c, codes, dcd, n * nk)) || (rc = sync(c))) return rc;
    return ANQI_OK;
}

int anqi_lrq_materialize(anqi_ctx* h, const float* coeff, const uint8_t* codes, uint64_t n, uint32_t nk,
                         uint32_t rankm, const float* mu, const float* basis, const float* codebook,
                         uint32_t code_size, uint32_t k, double radius_scale, float* thr) {
    if (!h || !coeff || !codes || !mu || !basis || !codebook || !thr) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    if (k < 1 || k > nk) return fail(c, ANQI_ERR_ARGS, "LRQ verifier is not ready for k=%u", k);
    Verifier v;
    int rc = load_verifier(c, v, coeff, codes, n, nk, rankm, mu, basis, codebook, code_size);
    TmpBuf out(c);
    if (!rc && !(rc = ensure(c, out, n * 4)) && !(rc = lrq_materialize_device(c, v, k, radius_scale, out.as<float>())))
        if (!(rc = d2h(c, thr, out, n * 4))) rc = sync(c);
    release(c, v.coeff);
    release(c, v.codes_t);
    release(c, v.mu);
    release(c, v.basis);
    release(c, v.codebook);
    return rc;
}

int anqi_verifier_load(anqi_ctx* h, const float* coeff, const uint8_t* codes, uint64_t n, uint32_t nk,
                       uint32_t rankm, const float* mu, const float* basis, const float* codebook,
                       uint32_t code_size) {
    if (!h || !coeff || !codes || !mu || !basis || !codebook) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    return load_verifier(c, c->vf, coeff, codes, n, nk, rankm, mu, basis, codebook, code_size);
}

}  // extern "C"
