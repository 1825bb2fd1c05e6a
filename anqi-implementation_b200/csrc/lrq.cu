// Rank-M + residual verifier codec: every CompactLrqVerifier form of the
// reference, and the analytic Rank-M model.
//
// Reference: CompactLrqVerifier::build / materialize_k, src/rknn_query.cpp:
// 679-753; encode_learned_residual (:482-513, policies nearest / floor /
// ceil); the packed-code layout of include/packed_code_array.h:8-63 (u2, u4,
// u8, u16); the radius modes of :144-186 -- rankm_resid_u{2,4,8,16}_lrq_*
// (learned codebook), rankm_resid_f32 (float residuals, bits 32), rankm_only
// (bits 0); AnalyticRankMVerifier::materialize_k (:515-601).
//
// The reference evaluates every sum in double without fused multiply-adds
// (-std=c++17 turns contraction off); every operation here is an explicit _rn
// intrinsic so nvcc cannot fuse them either.  On the device the codes are kept
// k-major (nk rows of n4 = round_up(n, 4) entries: u8 for up to 8 bits, u16
// for 16, f32 residuals for bits 32) so materializing one rank reads a
// contiguous column; four u8 codes arrive in one 32-bit load and are split
// with __byte_perm.
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "internal.h"

namespace anqi {

constexpr int kEncodeRows = 32;  // rows staged per block

__host__ __device__ inline bool packed_bits(uint32_t bits) { return bits == 2 || bits == 4 || bits == 8 || bits == 16; }

// packed_code_bytes (packed_code_array.h:14-18)
__host__ __device__ inline uint64_t packed_bytes(uint64_t count, uint32_t bits) {
    return packed_bits(bits) ? (count * bits + 7) / 8 : 0;
}

// get_packed_code (packed_code_array.h:45-61): little-endian sub-byte fields.
__device__ __forceinline__ uint32_t get_code(const uint8_t* data, uint64_t idx, uint32_t bits) {
    if (bits == 2) return (data[idx >> 2] >> ((uint32_t)(idx & 3u) * 2u)) & 3u;
    if (bits == 4) return (idx & 1u) ? (uint32_t)(data[idx >> 1] >> 4) : (uint32_t)(data[idx >> 1] & 15u);
    if (bits == 8) return data[idx];
    return (uint32_t)data[idx * 2] | ((uint32_t)data[idx * 2 + 1] << 8);
}

// encode_learned_residual (rknn_query.cpp:482-513): searches with the float
// value, compares the two neighbours of `nearest` in double.
__device__ __forceinline__ uint32_t encode_residual(double value, const float* __restrict__ c, uint32_t cs,
                                                    uint32_t policy) {
    const float v = __double2float_rn(value);
    if (policy == ANQI_LRQ_FLOOR) {  // upper_bound - 1, clamped to the first centre
        uint32_t lo = 0, hi = cs;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (v < __ldg(c + mid)) hi = mid;
            else lo = mid + 1;
        }
        return lo == 0 ? 0u : lo - 1;
    }
    uint32_t lo = 0, hi = cs;  // lower_bound: first centre >= v
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(c + mid) < v) lo = mid + 1;
        else hi = mid;
    }
    if (policy == ANQI_LRQ_CEIL) return lo == cs ? cs - 1 : lo;
    if (lo == 0) return 0u;
    if (lo == cs) return cs - 1;
    const double up = (double)__ldg(c + lo), dn = (double)__ldg(c + lo - 1);
    return fabs(__dsub_rn(up, value)) < fabs(__dsub_rn(value, dn)) ? lo : lo - 1;
}

// One thread per row; keys for kEncodeRows rows staged in shared memory, the
// rows' codes then packed in the reference's object-major layout (bits 2, 4,
// 8, 16), or their float residuals written (bits 32).
__global__ void lrq_encode_kernel(const float* __restrict__ keys, uint64_t n, uint32_t nk, uint32_t rankm,
                                  const float* __restrict__ mu, const float* __restrict__ basis,
                                  const float* __restrict__ codebook, uint32_t code_size, uint32_t bits,
                                  uint32_t policy, float* __restrict__ coeff, uint8_t* __restrict__ codes,
                                  float* __restrict__ resid) {
    extern __shared__ float sh[];
    float* s_keys = sh;                                  // kEncodeRows x nk (then their codes)
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
        if (bits != 0)
            for (uint32_t k = 0; k < nk; k++) {
                double recon = (double)s_mu[k];
                for (uint32_t m = 0; m < rankm; m++)
                    recon = __dadd_rn(recon, __dmul_rn((double)ci[m], (double)s_basis[m * nk + k]));
                const double residual = __dsub_rn((double)rk[k], recon);
                if (bits == 32) {
                    resid[(row0 + r) * nk + k] = __double2float_rn(residual);
                } else {
                    const uint32_t code = encode_residual(residual, codebook + (size_t)k * code_size, code_size, policy);
                    s_keys[(size_t)r * nk + k] = __uint_as_float(code);  // own row only: no other thread reads it
                }
            }
    }
    __syncthreads();
    if (!packed_bits(bits)) return;
    // set_packed_code (packed_code_array.h:20-43); whole bytes per block since
    // nk * bits is a multiple of 8 (checked on the host)
    const uint64_t bytes = (uint64_t)rows * nk * bits / 8;
    uint8_t* out = codes + row0 * nk * bits / 8;
    for (uint64_t t = threadIdx.x; t < bytes; t += blockDim.x) {
        uint32_t byte;
        if (bits == 16) {
            const uint32_t code = __float_as_uint(s_keys[t >> 1]);
            byte = (t & 1u) ? (code >> 8) & 255u : code & 255u;
        } else {
            const uint32_t per = 8 / bits, mask = (1u << bits) - 1u;
            byte = 0;
            for (uint32_t j = 0; j < per; j++) byte |= (__float_as_uint(s_keys[t * per + j]) & mask) << (j * bits);
        }
        out[t] = (uint8_t)byte;
    }
}

// Object-major packed codes / residuals (n x nk) -> k-major (nk x n4), 32 x 32 tiles.
template <class T>
__global__ void codes_transpose_kernel(const uint8_t* __restrict__ src, uint64_t n, uint32_t nk, uint64_t n4,
                                       uint32_t bits, T* __restrict__ dst) {
    __shared__ T tile[32][33];
    const uint64_t o0 = (uint64_t)blockIdx.x * 32;
    const uint32_t k0 = blockIdx.y * 32;
    for (uint32_t y = threadIdx.y; y < 32; y += blockDim.y) {
        const uint64_t o = o0 + y;
        const uint32_t k = k0 + threadIdx.x;
        T v = T(0);
        if (o < n && k < nk) {
            if constexpr (sizeof(T) == 4) v = reinterpret_cast<const T*>(src)[o * nk + k];
            else v = (T)get_code(src, o * nk + k, bits);
        }
        tile[y][threadIdx.x] = v;
    }
    __syncthreads();
    for (uint32_t y = threadIdx.y; y < 32; y += blockDim.y) {
        const uint32_t k = k0 + y;
        const uint64_t o = o0 + threadIdx.x;
        if (k < nk && o < n4) dst[(uint64_t)k * n4 + o] = tile[threadIdx.x][y];
    }
}

// thr[o] = f32(scale * (mu_k + sum_m c_om G_mk + residual)), clamped at 0
// unless the keys are signed (IP), four objects per thread.  Residual: none
// (bits 0), cb_k[code] (u8 / u16 codes), or the stored float (bits 32).
template <int kMode>  // 0 none, 1 u8 codes, 2 u16 codes, 3 float residuals
__global__ void lrq_materialize_kernel(const float* __restrict__ coeff, const void* __restrict__ codes_t, uint64_t n,
                                       uint64_t n4, uint32_t nk, uint32_t rankm, const float* __restrict__ mu,
                                       const float* __restrict__ basis, const float* __restrict__ codebook,
                                       uint32_t code_size, uint32_t k, double radius_scale, int signed_keys,
                                       float* __restrict__ thr) {
    __shared__ double s_g[16];
    if (threadIdx.x < rankm) s_g[threadIdx.x] = (double)basis[threadIdx.x * nk + k];
    __syncthreads();
    const double muk = (double)mu[k];
    const float* cb = codebook + (size_t)k * code_size;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; 4 * t < n;
         t += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t word = 0;
        if constexpr (kMode == 1) word = reinterpret_cast<const uint32_t*>(static_cast<const uint8_t*>(codes_t) + (uint64_t)k * n4)[t];
#pragma unroll
        for (uint32_t j = 0; j < 4; j++) {
            const uint64_t o = 4 * t + j;
            if (o >= n) break;
            const float* ci = coeff + o * rankm;
            double value = muk;
            for (uint32_t m = 0; m < rankm; m++) value = __dadd_rn(value, __dmul_rn((double)ci[m], s_g[m]));
            if constexpr (kMode == 1) {
                value = __dadd_rn(value, (double)__ldg(cb + __byte_perm(word, 0u, 0x4440u | j)));
            } else if constexpr (kMode == 2) {
                const uint32_t code = static_cast<const uint16_t*>(codes_t)[(uint64_t)k * n4 + o];
                value = __dadd_rn(value, (double)__ldg(cb + code));
            } else if constexpr (kMode == 3) {
                value = __dadd_rn(value, (double)static_cast<const float*>(codes_t)[(uint64_t)k * n4 + o]);
            }
            const double scaled = __dmul_rn(radius_scale, value);
            thr[o] = __double2float_rn(signed_keys ? scaled : (0.0 < scaled ? scaled : 0.0));
        }
    }
}

// AnalyticRankMVerifier::materialize_k (rknn_query.cpp:576-600): thr[i] =
// f32(max(0, scale * sum_m c_im * basis_m)), the basis computed on the host.
__global__ void analytic_materialize_kernel(const float* __restrict__ coeff, uint64_t n, uint32_t rankm,
                                            const double* __restrict__ pb, double radius_scale,
                                            float* __restrict__ thr) {
    __shared__ double s_b[16];
    if (threadIdx.x < rankm) s_b[threadIdx.x] = pb[threadIdx.x];
    __syncthreads();
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const float* ci = coeff + i * rankm;
        double value = 0.0;
        for (uint32_t m = 0; m < rankm; m++) value = __dadd_rn(value, __dmul_rn((double)ci[m], s_b[m]));
        const double scaled = __dmul_rn(radius_scale, value);
        thr[i] = __double2float_rn(0.0 < scaled ? scaled : 0.0);
    }
}

int lrq_materialize_device(Ctx* c, const Verifier& v, uint32_t k, double scale, float* d_out) {
    const uint64_t n4 = (v.n + 3) / 4 * 4;
    if (v.analytic) {
        // rknn_query.cpp:587-593: ratio = k / train_kmax (centred log) or k,
        // basis_0 = ratio^b0, basis_m = basis_{m-1} * log(ratio)
        const bool centered = (v.flags & 4u) != 0;
        const double ratio = centered ? (double)k / (double)v.train_kmax : (double)k;
        const double logk = std::log(ratio);
        double pb[16];
        pb[0] = std::pow(ratio, v.b0);
        for (uint32_t m = 1; m < v.rankm; m++) pb[m] = pb[m - 1] * logk;
        TmpBuf dpb(c);
        int rc = h2d(c, dpb, pb, v.rankm * sizeof(double));
        if (rc) return rc;
        const int blocks = (int)std::min<uint64_t>((v.n + 255) / 256, (uint64_t)c->sm_count * 8);
        analytic_materialize_kernel<<<std::max(blocks, 1), 256, 0, c->stream>>>(v.coeff.as<float>(), v.n, v.rankm,
                                                                                dpb.as<double>(), scale, d_out);
        ANQI_CUDA(c, cudaGetLastError());
        return sync(c);  // dpb is released on return
    }
    const int blocks = (int)std::min<uint64_t>((v.n / 4 + 256) / 256, (uint64_t)c->sm_count * 8);
    const int sk = v.signed_keys ? 1 : 0;
#define ANQI_MAT(MODE)                                                                                              \
    lrq_materialize_kernel<MODE><<<std::max(blocks, 1), 256, 0, c->stream>>>(                                       \
        v.coeff.as<float>(), v.codes_t.p, v.n, n4, v.nk, v.rankm, v.mu.as<float>(), v.basis.as<float>(),            \
        v.codebook.as<float>(), v.code_size, k - 1, scale, sk, d_out)
    if (v.bits == 0) ANQI_MAT(0);
    else if (v.bits <= 8) ANQI_MAT(1);
    else if (v.bits == 16) ANQI_MAT(2);
    else ANQI_MAT(3);
#undef ANQI_MAT
    ANQI_CUDA(c, cudaGetLastError());
    return ANQI_OK;
}

// CompactLrqVerifier::configure's checks (rknn_query.cpp:640-668) and the
// packed u2 / u4 divisibility rule (:687-693).
static int check_lrq_args(Ctx* c, uint64_t n, uint32_t nk, uint32_t rankm, uint32_t bits, uint32_t policy,
                          const float* codebook, uint32_t code_size) {
    const bool bits_ok = bits == 0 || bits == 32 || packed_bits(bits);
    const uint32_t want_cs = packed_bits(bits) ? (1u << bits) : 0u;
    if (n == 0 || nk == 0 || rankm == 0 || rankm > 16 || !bits_ok || code_size != want_cs || policy > 2 ||
        (packed_bits(bits) && !codebook))
        return fail(c, ANQI_ERR_ARGS,
                    "invalid CompactLrqVerifier configuration (n=%llu nk=%u rankm=%u bits=%u code_size=%u policy=%u)",
                    (unsigned long long)n, nk, rankm, bits, code_size, policy);
    if ((bits == 2 && nk % 4 != 0) || (bits == 4 && nk % 2 != 0))
        return fail(c, ANQI_ERR_FORMAT, "packed u%u verifier requires NK divisible by %u, got %u", bits,
                    bits == 2 ? 4u : 2u, nk);
    if (packed_bits(bits))
        for (uint32_t k = 0; k < nk; k++)
            for (uint32_t j = 1; j < code_size; j++)
                if (codebook[(size_t)k * code_size + j] < codebook[(size_t)k * code_size + j - 1])
                    return fail(c, ANQI_ERR_FORMAT, "LRQ codebook row is not sorted: k=%u", k + 1);
    return ANQI_OK;
}

static void release_verifier(Ctx* c, Verifier& v) {
    release(c, v.coeff);
    release(c, v.codes_t);
    release(c, v.mu);
    release(c, v.basis);
    release(c, v.codebook);
    v.loaded = false;
}

static int load_verifier(Ctx* c, Verifier& v, const float* coeff, const uint8_t* codes, const float* resid,
                         uint64_t n, uint32_t nk, uint32_t rankm, uint32_t bits, const float* mu, const float* basis,
                         const float* codebook, uint32_t code_size, bool signed_keys) {
    int rc = check_lrq_args(c, n, nk, rankm, bits, ANQI_LRQ_FLOOR, codebook, code_size);
    if (rc) return rc;
    if ((packed_bits(bits) && !codes) || (bits == 32 && !resid))
        return fail(c, ANQI_ERR_ARGS, "verifier load: codes (bits %u) missing", bits);
    v.loaded = false;
    v.analytic = false;
    v.n = n;
    v.nk = nk;
    v.rankm = rankm;
    v.bits = bits;
    v.code_size = code_size;
    v.signed_keys = signed_keys;
    const uint64_t n4 = (n + 3) / 4 * 4;
    const uint32_t esz = bits == 0 ? 0 : (bits <= 8 ? 1 : (bits == 16 ? 2 : 4));
    const uint64_t raw_bytes = bits == 32 ? n * nk * 4 : packed_bytes(n * nk, bits);
    TmpBuf raw(c);
    if ((rc = h2d(c, v.coeff, coeff, n * rankm * 4)) || (rc = h2d(c, v.mu, mu, nk * 4)) ||
        (rc = h2d(c, v.basis, basis, (size_t)rankm * nk * 4)))
        return rc;
    if (code_size && (rc = h2d(c, v.codebook, codebook, (size_t)nk * code_size * 4))) return rc;
    if (esz) {
        if ((rc = h2d(c, raw, bits == 32 ? static_cast<const void*>(resid) : codes, raw_bytes)) ||
            (rc = ensure(c, v.codes_t, nk * n4 * esz)))
            return rc;
        dim3 grid((unsigned)((n4 + 31) / 32), (nk + 31) / 32), block(32, 8);
        if (esz == 1)
            codes_transpose_kernel<uint8_t><<<grid, block, 0, c->stream>>>(raw.as<uint8_t>(), n, nk, n4, bits,
                                                                          v.codes_t.as<uint8_t>());
        else if (esz == 2)
            codes_transpose_kernel<uint16_t><<<grid, block, 0, c->stream>>>(raw.as<uint8_t>(), n, nk, n4, bits,
                                                                           v.codes_t.as<uint16_t>());
        else
            codes_transpose_kernel<float><<<grid, block, 0, c->stream>>>(raw.as<uint8_t>(), n, nk, n4, bits,
                                                                        v.codes_t.as<float>());
        ANQI_CUDA(c, cudaGetLastError());
    }
    if ((rc = sync(c))) return rc;
    v.loaded = true;
    return ANQI_OK;
}

static int lrq_encode(anqi_ctx* h, const float* keys, uint64_t n, uint32_t nk, uint32_t rankm, const float* mu,
                      const float* basis, const float* codebook, uint32_t code_size, uint32_t bits, uint32_t policy,
                      float* coeff, uint8_t* codes, float* resid) {
    if (!h || !keys || !mu || !basis || !coeff) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    int rc = check_lrq_args(c, n, nk, rankm, bits, policy, codebook, code_size);
    if (rc) return rc;
    if ((packed_bits(bits) && !codes) || (bits == 32 && !resid))
        return fail(c, ANQI_ERR_ARGS, "lrq_encode: output for bits %u missing", bits);
    const uint64_t code_bytes = packed_bytes(n * nk, bits), resid_bytes = bits == 32 ? n * nk * 4 : 0;
    TmpBuf dk(c), dmu(c), db(c), dcb(c), dco(c), dcd(c), dre(c);
    if ((rc = h2d(c, dk, keys, n * nk * 4)) || (rc = h2d(c, dmu, mu, nk * 4)) ||
        (rc = h2d(c, db, basis, (size_t)rankm * nk * 4)) || (rc = ensure(c, dco, n * rankm * 4)) ||
        (code_size && (rc = h2d(c, dcb, codebook, (size_t)nk * code_size * 4))) ||
        (code_bytes && (rc = ensure(c, dcd, code_bytes))) || (resid_bytes && (rc = ensure(c, dre, resid_bytes))))
        return rc;
    const size_t smem = ((size_t)kEncodeRows * nk + nk + (size_t)rankm * nk) * 4;
    if (smem > 200 * 1024) return fail(c, ANQI_ERR_ARGS, "nk too large for the encoder");
    ANQI_CUDA(c, cudaFuncSetAttribute(lrq_encode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const unsigned blocks = (unsigned)((n + kEncodeRows - 1) / kEncodeRows);
    lrq_encode_kernel<<<blocks, kEncodeRows, smem, c->stream>>>(
        dk.as<float>(), n, nk, rankm, dmu.as<float>(), db.as<float>(), dcb.as<float>(), code_size, bits, policy,
        dco.as<float>(), dcd.as<uint8_t>(), dre.as<float>());
    ANQI_CUDA(c, cudaGetLastError());
    if ((rc = d2h(c, coeff, dco, n * rankm * 4)) || (code_bytes && (rc = d2h(c, codes, dcd, code_bytes))) ||
        (resid_bytes && (rc = d2h(c, resid, dre, resid_bytes))) || (rc = sync(c)))
        return rc;
    return ANQI_OK;
}

static int lrq_materialize(anqi_ctx* h, const float* coeff, const uint8_t* codes, const float* resid, uint64_t n,
                           uint32_t nk, uint32_t rankm, uint32_t bits, const float* mu, const float* basis,
                           const float* codebook, uint32_t code_size, uint32_t k, double radius_scale,
                           int signed_keys, float* thr) {
    if (!h || !coeff || !mu || !basis || !thr) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    if (k < 1 || k > nk) return fail(c, ANQI_ERR_ARGS, "LRQ verifier is not ready for k=%u", k);
    Verifier v;
    int rc = load_verifier(c, v, coeff, codes, resid, n, nk, rankm, bits, mu, basis, codebook, code_size,
                           signed_keys != 0);
    TmpBuf out(c);
    if (!rc && !(rc = ensure(c, out, n * 4)) && !(rc = lrq_materialize_device(c, v, k, radius_scale, out.as<float>())))
        if (!(rc = d2h(c, thr, out, n * 4))) rc = sync(c);
    release_verifier(c, v);
    return rc;
}

// AnalyticRankMVerifier::load's header checks (rknn_query.cpp:536-548).
static int check_analytic(Ctx* c, uint64_t n, uint32_t rankm, uint32_t train_kmax, uint32_t fit_kmin,
                          uint32_t flags, double b0) {
    if (n == 0 || rankm == 0 || rankm > 16 || train_kmax < 1 || fit_kmin < 1 || fit_kmin > train_kmax ||
        (flags != 3u && flags != 7u) || !std::isfinite(b0))
        return fail(c, ANQI_ERR_FORMAT, "analytic Rank-M header mismatch: train_kmax=%u rankm=%u fit_kmin=%u flags=%u",
                    train_kmax, rankm, fit_kmin, flags);
    return ANQI_OK;
}

}  // namespace anqi

using namespace anqi;

extern "C" {

int anqi_lrq_encode(anqi_ctx* h, const float* keys, uint64_t n, uint32_t nk, uint32_t rankm, const float* mu,
                    const float* basis, const float* codebook, uint32_t code_size, float* coeff, uint8_t* codes) {
    return lrq_encode(h, keys, n, nk, rankm, mu, basis, codebook, code_size, 8, ANQI_LRQ_FLOOR, coeff, codes, nullptr);
}

int anqi_lrq_encode_bits(anqi_ctx* h, const float* keys, uint64_t n, uint32_t nk, uint32_t rankm, const float* mu,
                         const float* basis, const float* codebook, uint32_t code_size, uint32_t bits,
                         uint32_t policy, float* coeff, uint8_t* codes, float* residual) {
    return lrq_encode(h, keys, n, nk, rankm, mu, basis, codebook, code_size, bits, policy, coeff, codes, residual);
}

int anqi_lrq_materialize(anqi_ctx* h, const float* coeff, const uint8_t* codes, uint64_t n, uint32_t nk,
                         uint32_t rankm, const float* mu, const float* basis, const float* codebook,
                         uint32_t code_size, uint32_t k, double radius_scale, float* thr) {
    if (!codes) return ANQI_ERR_ARGS;
    return lrq_materialize(h, coeff, codes, nullptr, n, nk, rankm, 8, mu, basis, codebook, code_size, k, radius_scale,
                           0, thr);
}

int anqi_lrq_materialize_bits(anqi_ctx* h, const float* coeff, const uint8_t* codes, const float* residual,
                              uint64_t n, uint32_t nk, uint32_t rankm, uint32_t bits, const float* mu,
                              const float* basis, const float* codebook, uint32_t code_size, uint32_t k,
                              double radius_scale, int signed_keys, float* thr) {
    return lrq_materialize(h, coeff, codes, residual, n, nk, rankm, bits, mu, basis, codebook, code_size, k,
                           radius_scale, signed_keys, thr);
}

int anqi_verifier_load(anqi_ctx* h, const float* coeff, const uint8_t* codes, uint64_t n, uint32_t nk,
                       uint32_t rankm, const float* mu, const float* basis, const float* codebook,
                       uint32_t code_size) {
    if (!h || !coeff || !codes || !mu || !basis || !codebook) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    return load_verifier(c, c->vf, coeff, codes, nullptr, n, nk, rankm, 8, mu, basis, codebook, code_size, false);
}

int anqi_verifier_load_bits(anqi_ctx* h, const float* coeff, const uint8_t* codes, const float* residual, uint64_t n,
                            uint32_t nk, uint32_t rankm, uint32_t bits, const float* mu, const float* basis,
                            const float* codebook, uint32_t code_size, int signed_keys) {
    if (!h || !coeff || !mu || !basis) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    return load_verifier(c, c->vf, coeff, codes, residual, n, nk, rankm, bits, mu, basis, codebook, code_size,
                         signed_keys != 0);
}

int anqi_analytic_rankm_materialize(anqi_ctx* h, const float* coeff, uint64_t n, uint32_t rankm,
                                    uint32_t train_kmax, uint32_t fit_kmin, uint32_t flags, double b0, uint32_t k,
                                    double radius_scale, float* thr) {
    if (!h || !coeff || !thr || k == 0) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    int rc = check_analytic(c, n, rankm, train_kmax, fit_kmin, flags, b0);
    if (rc) return rc;
    Verifier v;
    v.analytic = true;
    v.n = n;
    v.rankm = rankm;
    v.train_kmax = train_kmax;
    v.flags = flags;
    v.b0 = b0;
    TmpBuf out(c);
    if (!(rc = h2d(c, v.coeff, coeff, n * rankm * 4)) && !(rc = ensure(c, out, n * 4)) &&
        !(rc = lrq_materialize_device(c, v, k, radius_scale, out.as<float>())))
        if (!(rc = d2h(c, thr, out, n * 4))) rc = sync(c);
    release_verifier(c, v);
    return rc;
}

int anqi_verifier_load_analytic(anqi_ctx* h, const float* coeff, uint64_t n, uint32_t rankm, uint32_t train_kmax,
                                uint32_t fit_kmin, uint32_t flags, double b0) {
    if (!h || !coeff) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    int rc = check_analytic(c, n, rankm, train_kmax, fit_kmin, flags, b0);
    if (rc) return rc;
    Verifier& v = c->vf;
    v.loaded = false;
    v.analytic = true;
    v.n = n;
    v.rankm = rankm;
    v.nk = 0xFFFFFFFFu;  // any rank
    v.train_kmax = train_kmax;
    v.flags = flags;
    v.b0 = b0;
    v.signed_keys = false;
    if ((rc = h2d(c, v.coeff, coeff, n * rankm * 4)) || (rc = sync(c))) return rc;
    v.loaded = true;
    return ANQI_OK;
}

}  // extern "C"
