/* Test infrastructure only -- never linked into or called from the product.
 *
 * Exact reverse-kNN ground truth on the host CPU, for the benchmark's
 * reference arm, which must not touch the GPU library: the same outputs as the
 * reference's tools/dataset_gt.cpp (thresholds mode :206-262, ground-truth mode
 * :270-313), at a cost that fits a benchmark run at n = 1M.
 *
 *   gt_cpu BASE.fbin QUERY.fbin HINTS.rec OUT_PREFIX K KS THREADS
 *
 * BASE / QUERY: [u32 n][u32 d][f32 ...].  HINTS: the AKNN source records
 * (n x K' {u32 id, f32 key}, K' >= K, e.g. _baseknn_aknn.rec); each row's K
 * hint ids bound its exact K-th key from above.  KS: comma list of ranks
 * k <= K.  Writes, for every k in KS:
 *   OUT_PREFIX_rknn_gt_k{k}.bin   [u32 nq][(nq+1) u32 off][u32 ids][f32 keys],
 *                                 per query ascending (key, id)   (dataset_gt.cpp:291-307)
 *   OUT_PREFIX_k{k}.rk            [u32 n][u32 k][f32 n] rank-k keys (dataset_gt.cpp:248-252)
 * and prints one JSON line of timings.
 *
 * Exactness.  dataset_gt computes key = |a|^2 + |b|^2 - 2 IP(a, b) in FP32 in
 * its AVX-512 order.  This program accepts only inputs on which every such
 * quantity is an exactly representable integer: all values integers with
 * |v| <= 256 and 2 d max|v|^2 < 2^24.  There every product and partial sum is
 * an integer below 2^24, so any summation order gives the same FP32 bits, and
 * BF16 holds every value exactly.  Inner products then run as AMX BF16 tiles
 * (TDPBF16PS, FP32 accumulation) where the CPU and kernel allow it, else as
 * AVX-512 FP32 FMAs; both are bit-exact with the reference's keys.  Other
 * inputs exit with status 3 (use dataset_gt there).
 *
 * Algorithm.  Thresholds: for each row i, bound_i = max key(i, hint) over its
 * K hints >= its exact K-th key; every pair (i, j != i) with key <= bound_i is
 * kept and the row's kept keys are sorted: the k-th smallest is r_k(i).
 * Ground truth: every (q, j) with key(q, j) <= r_k(j), sorted by (key, id).
 */
#define _GNU_SOURCE
#include <cpuid.h>
#include <immintrin.h>
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/syscall.h>
#include <time.h>
#include <unistd.h>

#define ARCH_REQ_XCOMP_PERM 0x1023
#define XFEATURE_XTILEDATA 18
#define PANEL 1024 /* rows per panel (A panel 1024 x D bf16 stays in L2) */

typedef struct {
    float key;
    uint32_t id;
} kv_t;

typedef struct {
    kv_t* v;
    uint32_t n, cap;
} kvlist_t;

static void die(const char* msg) {
    fprintf(stderr, "[gt_cpu] %s\n", msg);
    exit(3);
}

static void kv_push(kvlist_t* l, float key, uint32_t id) {
    if (l->n == l->cap) {
        l->cap = l->cap ? 2 * l->cap : 256;
        l->v = (kv_t*)realloc(l->v, (size_t)l->cap * sizeof(kv_t));
        if (!l->v) die("out of memory");
    }
    l->v[l->n].key = key;
    l->v[l->n].id = id;
    l->n++;
}

static int cmp_kv(const void* a, const void* b) {
    const kv_t* x = (const kv_t*)a;
    const kv_t* y = (const kv_t*)b;
    if (x->key < y->key) return -1;
    if (x->key > y->key) return 1;
    return (x->id > y->id) - (x->id < y->id);
}

static double now_s(void) {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec + 1e-9 * t.tv_nsec;
}

static float* read_fbin(const char* path, uint32_t* n, uint32_t* d) {
    FILE* f = fopen(path, "rb");
    if (!f) die("cannot open an fbin input");
    uint32_t h[2];
    if (fread(h, 4, 2, f) != 2) die("short fbin header");
    *n = h[0];
    *d = h[1];
    float* x = (float*)malloc((size_t)h[0] * h[1] * 4 + 64);
    if (!x || fread(x, 4, (size_t)h[0] * h[1], f) != (size_t)h[0] * h[1]) die("short fbin body");
    fclose(f);
    return x;
}

/* Integers with |v| <= 256, and 2 d max^2 < 2^24: every key exact in FP32. */
static int exact_inputs(const float* x, size_t m, uint32_t d, double* vmax) {
    for (size_t i = 0; i < m; i++) {
        const float v = x[i];
        if (!(fabsf(v) <= 256.0f) || v != rintf(v)) return 0;
        if (fabs((double)v) > *vmax) *vmax = fabs((double)v);
    }
    return 2.0 * d * (*vmax) * (*vmax) < 16777216.0;
}

static float dot_exact(const float* a, const float* b, uint32_t d) {
    float s = 0.0f; /* exact: integer products and sums below 2^24 */
    for (uint32_t t = 0; t < d; t++) s += a[t] * b[t];
    return s;
}

/* ------------------------------------------------------------------ AMX */

typedef struct {
    uint8_t palette_id, start_row, reserved[14];
    uint16_t colsb[16];
    uint8_t rows[16];
} tilecfg_t;

static int amx_available(void) {
    unsigned a, b, c, d;
    if (!__get_cpuid_count(7, 0, &a, &b, &c, &d)) return 0;
    if (!((d >> 22) & 1u) || !((d >> 24) & 1u)) return 0; /* AMX-BF16, AMX-TILE */
    if (syscall(SYS_arch_prctl, ARCH_REQ_XCOMP_PERM, XFEATURE_XTILEDATA) != 0) return 0;
    return 1;
}

__attribute__((target("amx-tile,amx-bf16"))) static void amx_config(void) {
    tilecfg_t cfg;
    memset(&cfg, 0, sizeof cfg);
    cfg.palette_id = 1;
    for (int t = 0; t < 8; t++) {
        cfg.rows[t] = 16;
        cfg.colsb[t] = 64;
    }
    _tile_loadconfig(&cfg);
}

/* Inner products of 32 A rows (bf16, row stride Dp) with 32 packed B columns
 * (two 16-column blocks of nkc 1 KB VNNI tiles each) into C (32 x 32 floats). */
__attribute__((target("amx-tile,amx-bf16"))) static void amx_block(const uint16_t* A, size_t Dp, const uint16_t* B0,
                                                                   const uint16_t* B1, uint32_t nkc, float* C) {
    _tile_zero(0);
    _tile_zero(1);
    _tile_zero(2);
    _tile_zero(3);
    for (uint32_t kc = 0; kc < nkc; kc++) {
        _tile_loadd(4, A + kc * 32, (long)(Dp * 2));
        _tile_loadd(5, A + 16 * Dp + kc * 32, (long)(Dp * 2));
        _tile_loadd(6, B0 + (size_t)kc * 512, 64);
        _tile_loadd(7, B1 + (size_t)kc * 512, 64);
        _tile_dpbf16ps(0, 4, 6);
        _tile_dpbf16ps(1, 4, 7);
        _tile_dpbf16ps(2, 5, 6);
        _tile_dpbf16ps(3, 5, 7);
    }
    _tile_stored(0, C, 128);
    _tile_stored(1, C + 16, 128);
    _tile_stored(2, C + 16 * 32, 128);
    _tile_stored(3, C + 16 * 32 + 16, 128);
}

__attribute__((target("amx-tile"))) static void amx_release(void) { _tile_release(); }

/* AVX-512 FP32 form of amx_block on the FP32 rows (exact on accepted inputs). */
__attribute__((target("avx512f"))) static void fma_block(const float* A, size_t lda, uint32_t na, const float* B,
                                                         size_t ldb, uint32_t nb, uint32_t d, float* C) {
    for (uint32_t r = 0; r < 32; r++) {
        const float* a = A + (size_t)(r < na ? r : 0) * lda;
        for (uint32_t c = 0; c < 32; c += 8) {
            __m512 acc[8];
            for (int u = 0; u < 8; u++) acc[u] = _mm512_setzero_ps();
            for (uint32_t t = 0; t < d; t += 16) {
                const __m512 av = _mm512_loadu_ps(a + t);
                for (int u = 0; u < 8; u++) {
                    const uint32_t cc = c + u < nb ? c + u : 0;
                    acc[u] = _mm512_fmadd_ps(av, _mm512_loadu_ps(B + (size_t)cc * ldb + t), acc[u]);
                }
            }
            for (int u = 0; u < 8; u++) C[r * 32 + c + u] = _mm512_reduce_add_ps(acc[u]);
        }
    }
}

/* Row-major bf16 copy (rows padded to Dp, zero-filled). */
static uint16_t* to_bf16_rows(const float* x, uint32_t n, uint32_t d, uint32_t n_pad, size_t Dp) {
    uint16_t* a = (uint16_t*)aligned_alloc(64, (size_t)n_pad * Dp * 2 + 64);
    if (!a) die("out of memory");
    memset(a, 0, (size_t)n_pad * Dp * 2);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++)
        for (uint32_t t = 0; t < d; t++) {
            uint32_t u;
            memcpy(&u, &x[(size_t)i * d + t], 4);
            a[(size_t)i * Dp + t] = (uint16_t)(u >> 16); /* exact: the value is bf16-representable */
        }
    return a;
}

/* VNNI tiles: for 16-column block J and 32-deep chunk kc, 16 rows r x 16
 * columns c x 2: element (r, c, p) = x[16J + c][32 kc + 2r + p]. */
static uint16_t* to_bf16_vnni(const uint16_t* rows, uint32_t n_pad, size_t Dp) {
    const uint32_t nkc = (uint32_t)(Dp / 32), nblk = n_pad / 16;
    uint16_t* b = (uint16_t*)aligned_alloc(64, (size_t)n_pad * Dp * 2 + 64);
    if (!b) die("out of memory");
#pragma omp parallel for schedule(static)
    for (int64_t J = 0; J < (int64_t)nblk; J++)
        for (uint32_t kc = 0; kc < nkc; kc++) {
            uint16_t* t = b + ((size_t)J * nkc + kc) * 512;
            for (uint32_t r = 0; r < 16; r++)
                for (uint32_t c = 0; c < 16; c++)
                    for (uint32_t p = 0; p < 2; p++)
                        t[(r * 16 + c) * 2 + p] = rows[((size_t)J * 16 + c) * Dp + kc * 32 + 2 * r + p];
        }
    return b;
}

typedef struct {
    const float* a; /* FP32 rows (FP32 path) */
    const float* b;
    uint32_t na, nb, d;
    const uint16_t* a16; /* bf16 rows / packed columns (AMX path) */
    const uint16_t* b16;
    size_t Dp;
    uint32_t nkc;
    int amx;
} pairs_t;

/* C = IP(rows r0..r0+31, columns c0..c0+31), out-of-range entries unspecified. */
static void ip_block(const pairs_t* P, uint32_t r0, uint32_t c0, float* C) {
    if (P->amx) {
        const uint16_t* B0 = P->b16 + (size_t)(c0 / 16) * P->nkc * 512;
        amx_block(P->a16 + (size_t)r0 * P->Dp, P->Dp, B0, B0 + (size_t)P->nkc * 512, P->nkc, C);
    } else {
        fma_block(P->a + (size_t)r0 * P->d, P->d, P->na - r0 < 32 ? P->na - r0 : 32, P->b + (size_t)c0 * P->d, P->d,
                  P->nb - c0 < 32 ? P->nb - c0 : 32, P->d, C);
    }
}

/* ------------------------------------------------- thresholds (top-K keys) */

__attribute__((target("avx512f"))) static void keep_rows(const float* C, uint32_t r0, uint32_t c0, uint32_t n,
                                                         const float* norm, const float* bound, kvlist_t* lists,
                                                         uint32_t list_base) {
    const uint32_t nc = n - c0 < 32 ? n - c0 : 32;
    const __mmask16 cm0 = nc >= 16 ? 0xFFFF : (__mmask16)((1u << nc) - 1u);
    const __mmask16 cm1 = nc >= 32 ? 0xFFFF : (nc > 16 ? (__mmask16)((1u << (nc - 16)) - 1u) : 0);
    const __m512 nj0 = _mm512_maskz_loadu_ps(cm0, norm + c0), nj1 = _mm512_maskz_loadu_ps(cm1, norm + c0 + 16);
    const __m512 two = _mm512_set1_ps(2.0f);
    for (uint32_t r = 0; r < 32; r++) {
        const uint32_t i = r0 + r;
        if (i >= n) break;
        const __m512 ni = _mm512_set1_ps(norm[i]), bi = _mm512_set1_ps(bound[i]);
        /* dataset_gt.cpp:223: key = bnorm[ti] + nj - 2 ip */
        const __m512 k0 = _mm512_sub_ps(_mm512_add_ps(ni, nj0), _mm512_mul_ps(two, _mm512_loadu_ps(C + r * 32)));
        const __m512 k1 = _mm512_sub_ps(_mm512_add_ps(ni, nj1), _mm512_mul_ps(two, _mm512_loadu_ps(C + r * 32 + 16)));
        uint32_t m = (uint32_t)_mm512_mask_cmp_ps_mask(cm0, k0, bi, _CMP_LE_OQ) |
                     ((uint32_t)_mm512_mask_cmp_ps_mask(cm1, k1, bi, _CMP_LE_OQ) << 16);
        if (i >= c0 && i < c0 + 32) m &= ~(1u << (i - c0)); /* self excluded (dataset_gt.cpp:220) */
        if (!m) continue;
        float kk[32];
        _mm512_storeu_ps(kk, k0);
        _mm512_storeu_ps(kk + 16, k1);
        while (m) {
            const uint32_t c = (uint32_t)__builtin_ctz(m);
            m &= m - 1;
            kv_push(&lists[i - list_base], kk[c], c0 + c);
        }
    }
}

static void thresholds(const pairs_t* P, const float* norm, const float* bound, const uint32_t* ks, uint32_t nks,
                       float** rk, uint64_t* kept) {
    const uint32_t n = P->na;
    const uint32_t npanel = (n + PANEL - 1) / PANEL;
    uint64_t kept_total = 0;
#pragma omp parallel reduction(+ : kept_total)
    {
        if (P->amx) amx_config();
        float* C = (float*)aligned_alloc(64, 32 * 32 * 4);
        kvlist_t* lists = (kvlist_t*)calloc(PANEL, sizeof(kvlist_t));
#pragma omp for schedule(dynamic, 1)
        for (int64_t pi = 0; pi < (int64_t)npanel; pi++) {
            const uint32_t p0 = (uint32_t)pi * PANEL, p1 = p0 + PANEL < n ? p0 + PANEL : n;
            for (uint32_t r = 0; r < p1 - p0; r++) lists[r].n = 0;
            for (uint32_t c0 = 0; c0 < n; c0 += 32)
                for (uint32_t r0 = p0; r0 < p1; r0 += 32) {
                    ip_block(P, r0, c0, C);
                    keep_rows(C, r0, c0, n, norm, bound, lists, p0);
                }
            for (uint32_t r = 0; r < p1 - p0; r++) {
                kvlist_t* l = &lists[r];
                qsort(l->v, l->n, sizeof(kv_t), cmp_kv);
                kept_total += l->n;
                for (uint32_t t = 0; t < nks; t++) {
                    if (l->n < ks[t]) die("a row kept fewer keys than its rank (bad hints)");
                    rk[t][p0 + r] = l->v[ks[t] - 1].key;
                }
            }
        }
        for (uint32_t r = 0; r < PANEL; r++) free(lists[r].v);
        free(lists);
        free(C);
        if (P->amx) amx_release();
    }
    *kept = kept_total;
}

/* ------------------------------------------------------ reverse-kNN sets */

__attribute__((target("avx512f"))) static void keep_queries(const float* C, uint32_t r0, uint32_t c0, uint32_t nq,
                                                            uint32_t n, const float* qnorm, const float* bnorm,
                                                            float* const* rk, uint32_t nks, const float* rmax,
                                                            kvlist_t* lists, uint32_t list_base) {
    const uint32_t nc = n - c0 < 32 ? n - c0 : 32;
    const __mmask16 cm0 = nc >= 16 ? 0xFFFF : (__mmask16)((1u << nc) - 1u);
    const __mmask16 cm1 = nc >= 32 ? 0xFFFF : (nc > 16 ? (__mmask16)((1u << (nc - 16)) - 1u) : 0);
    const __m512 nj0 = _mm512_maskz_loadu_ps(cm0, bnorm + c0), nj1 = _mm512_maskz_loadu_ps(cm1, bnorm + c0 + 16);
    const __m512 r0v = _mm512_maskz_loadu_ps(cm0, rmax + c0), r1v = _mm512_maskz_loadu_ps(cm1, rmax + c0 + 16);
    const __m512 two = _mm512_set1_ps(2.0f);
    for (uint32_t r = 0; r < 32; r++) {
        const uint32_t q = r0 + r;
        if (q >= nq) break;
        const __m512 qn = _mm512_set1_ps(qnorm[q]);
        /* dataset_gt.cpp:287: key = qn + bnorm[j] - 2 ip */
        const __m512 k0 = _mm512_sub_ps(_mm512_add_ps(qn, nj0), _mm512_mul_ps(two, _mm512_loadu_ps(C + r * 32)));
        const __m512 k1 = _mm512_sub_ps(_mm512_add_ps(qn, nj1), _mm512_mul_ps(two, _mm512_loadu_ps(C + r * 32 + 16)));
        uint32_t m = (uint32_t)_mm512_mask_cmp_ps_mask(cm0, k0, r0v, _CMP_LE_OQ) |
                     ((uint32_t)_mm512_mask_cmp_ps_mask(cm1, k1, r1v, _CMP_LE_OQ) << 16);
        if (!m) continue;
        float kk[32];
        _mm512_storeu_ps(kk, k0);
        _mm512_storeu_ps(kk + 16, k1);
        while (m) {
            const uint32_t c = (uint32_t)__builtin_ctz(m);
            m &= m - 1;
            const uint32_t j = c0 + c;
            for (uint32_t t = 0; t < nks; t++)
                if (kk[c] <= rk[t][j]) kv_push(&lists[(size_t)(q - list_base) * nks + t], kk[c], j);
        }
    }
}

static void write_csr(const char* path, uint32_t nq, kvlist_t* lists, uint32_t nks, uint32_t t) {
    FILE* f = fopen(path, "wb");
    if (!f) die("cannot open a ground-truth output");
    uint32_t* off = (uint32_t*)malloc((size_t)(nq + 1) * 4);
    off[0] = 0;
    for (uint32_t q = 0; q < nq; q++) off[q + 1] = off[q] + lists[(size_t)q * nks + t].n;
    fwrite(&nq, 4, 1, f);
    fwrite(off, 4, (size_t)nq + 1, f);
    for (uint32_t q = 0; q < nq; q++) {
        const kvlist_t* l = &lists[(size_t)q * nks + t];
        for (uint32_t i = 0; i < l->n; i++) fwrite(&l->v[i].id, 4, 1, f);
    }
    for (uint32_t q = 0; q < nq; q++) {
        const kvlist_t* l = &lists[(size_t)q * nks + t];
        for (uint32_t i = 0; i < l->n; i++) fwrite(&l->v[i].key, 4, 1, f);
    }
    if (fclose(f) != 0) die("write failed");
    free(off);
}

int main(int argc, char** argv) {
    if (argc != 8) {
        fprintf(stderr, "usage: gt_cpu BASE.fbin QUERY.fbin HINTS.rec OUT_PREFIX K KS THREADS\n");
        return 2;
    }
    const uint32_t K = (uint32_t)strtoul(argv[5], NULL, 10);
    const int threads = atoi(argv[7]);
    uint32_t ks[16], nks = 0;
    for (char* s = argv[6]; *s && nks < 16;) {
        ks[nks++] = (uint32_t)strtoul(s, &s, 10);
        if (*s == ',') s++;
    }
    if (threads > 0) omp_set_num_threads(threads);
    const double t_all = now_s();
    uint32_t n, d, nq, dq;
    float* base = read_fbin(argv[1], &n, &d);
    float* query = read_fbin(argv[2], &nq, &dq);
    if (dq != d || K == 0 || K >= n || nks == 0) die("bad sizes");
    for (uint32_t t = 0; t < nks; t++)
        if (ks[t] == 0 || ks[t] > K) die("every k must be in 1..K");
    double vmax = 0.0;
    if (!exact_inputs(base, (size_t)n * d, d, &vmax) || !exact_inputs(query, (size_t)nq * d, d, &vmax))
        die("inputs are not small integers (|v| <= 256, 2 d max^2 < 2^24): keys would not be exact; use dataset_gt");

    /* norms and hint bounds */
    float* bnorm = (float*)malloc((size_t)n * 4 + 64);
    float* qnorm = (float*)malloc((size_t)nq * 4 + 64);
    float* bound = (float*)malloc((size_t)n * 4 + 64);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) bnorm[i] = dot_exact(base + (size_t)i * d, base + (size_t)i * d, d);
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < (int64_t)nq; q++) qnorm[q] = dot_exact(query + (size_t)q * d, query + (size_t)q * d, d);
    {
        FILE* f = fopen(argv[3], "rb");
        if (!f) die("cannot open the hints");
        fseek(f, 0, SEEK_END);
        const long bytes = ftell(f);
        fseek(f, 0, SEEK_SET);
        if (bytes <= 0 || bytes % ((long)n * 8) != 0) die("hints file size is not n x K' records");
        const uint32_t kh = (uint32_t)(bytes / ((long)n * 8));
        if (kh < K) die("hints hold fewer than K ids per row");
        uint32_t* rec = (uint32_t*)malloc((size_t)bytes);
        if (fread(rec, 1, (size_t)bytes, f) != (size_t)bytes) die("short hints");
        fclose(f);
#pragma omp parallel
        {
            /* stamp[j] = row + 1 once row's hints named j: duplicates detected in O(K) */
            uint32_t* stamp = (uint32_t*)calloc(n, 4);
#pragma omp for schedule(static)
            for (int64_t i = 0; i < (int64_t)n; i++) {
                float b = -INFINITY;
                int ok = 1;
                for (uint32_t t = 0; t < K; t++) {
                    const uint32_t j = rec[((size_t)i * kh + t) * 2];
                    if (j >= n || j == (uint32_t)i || stamp[j] == (uint32_t)i + 1u) {
                        ok = 0;
                        break;
                    }
                    stamp[j] = (uint32_t)i + 1u;
                    const float ip = dot_exact(base + (size_t)i * d, base + (size_t)j * d, d);
                    const float key = (bnorm[i] + bnorm[j]) - 2.0f * ip;
                    if (key > b) b = key;
                }
                /* K distinct other rows bound the exact K-th key; without them keep every pair */
                bound[i] = ok ? b : INFINITY;
            }
            free(stamp);
        }
        free(rec);
    }

    const int amx = getenv("GT_CPU_NO_AMX") ? 0 : amx_available();
    const size_t Dp = ((size_t)d + 31) / 32 * 32;
    const uint32_t n_pad = (n + 31) / 32 * 32, nq_pad = (nq + 31) / 32 * 32;
    pairs_t P;
    memset(&P, 0, sizeof P);
    P.amx = amx;
    P.d = d;
    P.Dp = Dp;
    P.nkc = (uint32_t)(Dp / 32);
    float* base_pad = NULL;
    float* query_pad = NULL;
    uint16_t *b_rows = NULL, *b_vnni = NULL, *q_rows = NULL;
    if (amx) {
        b_rows = to_bf16_rows(base, n, d, n_pad, Dp);
        b_vnni = to_bf16_vnni(b_rows, n_pad, Dp);
        q_rows = to_bf16_rows(query, nq, d, nq_pad, Dp);
    } else {
        /* FP32 rows padded to a multiple of 16 floats for the FMA loop */
        const uint32_t dp = (d + 15) / 16 * 16;
        base_pad = (float*)calloc((size_t)n * dp + 16, 4);
        query_pad = (float*)calloc((size_t)nq * dp + 16, 4);
        for (size_t i = 0; i < n; i++) memcpy(base_pad + i * dp, base + i * d, (size_t)d * 4);
        for (size_t i = 0; i < nq; i++) memcpy(query_pad + i * dp, query + i * d, (size_t)d * 4);
        P.d = dp;
    }

    /* thresholds: rows = base, columns = base */
    float* rk[16];
    for (uint32_t t = 0; t < nks; t++) rk[t] = (float*)malloc((size_t)n * 4 + 64);
    const double t_thr = now_s();
    P.na = n;
    P.nb = n;
    P.a = base_pad;
    P.b = base_pad;
    P.a16 = b_rows;
    P.b16 = b_vnni;
    uint64_t kept = 0;
    thresholds(&P, bnorm, bound, ks, nks, rk, &kept);
    const double thr_s = now_s() - t_thr;

    /* reverse-kNN sets: rows = queries, columns = base */
    const double t_gt = now_s();
    float* rmax = (float*)malloc((size_t)n * 4 + 64);
    for (uint32_t j = 0; j < n; j++) {
        float m = rk[0][j];
        for (uint32_t t = 1; t < nks; t++) m = rk[t][j] > m ? rk[t][j] : m;
        rmax[j] = m;
    }
    kvlist_t* lists = (kvlist_t*)calloc((size_t)nq * nks, sizeof(kvlist_t));
    P.na = nq;
    P.a = query_pad;
    P.a16 = q_rows;
    const uint32_t qpanel = 64;
    const uint32_t nqp = (nq + qpanel - 1) / qpanel;
#pragma omp parallel
    {
        if (amx) amx_config();
        float* C = (float*)aligned_alloc(64, 32 * 32 * 4);
#pragma omp for schedule(dynamic, 1)
        for (int64_t pi = 0; pi < (int64_t)nqp; pi++) {
            const uint32_t p0 = (uint32_t)pi * qpanel, p1 = p0 + qpanel < nq ? p0 + qpanel : nq;
            for (uint32_t c0 = 0; c0 < n; c0 += 32)
                for (uint32_t r0 = p0; r0 < p1; r0 += 32) {
                    ip_block(&P, r0, c0, C);
                    keep_queries(C, r0, c0, p1, n, qnorm, bnorm, rk, nks, rmax, lists, 0);
                }
            for (uint32_t q = p0; q < p1; q++)
                for (uint32_t t = 0; t < nks; t++) {
                    kvlist_t* l = &lists[(size_t)q * nks + t];
                    qsort(l->v, l->n, sizeof(kv_t), cmp_kv);
                }
        }
        free(C);
        if (amx) amx_release();
    }
    const double gt_s = now_s() - t_gt;

    char path[4096];
    uint64_t pairs[16];
    for (uint32_t t = 0; t < nks; t++) {
        snprintf(path, sizeof path, "%s_rknn_gt_k%u.bin", argv[4], ks[t]);
        write_csr(path, nq, lists, nks, t);
        pairs[t] = 0;
        for (uint32_t q = 0; q < nq; q++) pairs[t] += lists[(size_t)q * nks + t].n;
        snprintf(path, sizeof path, "%s_k%u.rk", argv[4], ks[t]);
        FILE* f = fopen(path, "wb");
        if (!f) die("cannot open a threshold output");
        const uint32_t hdr[2] = {n, ks[t]};
        fwrite(hdr, 4, 2, f);
        fwrite(rk[t], 4, n, f);
        if (fclose(f) != 0) die("write failed");
    }
    printf("{\"n\": %u, \"nq\": %u, \"d\": %u, \"K\": %u, \"path\": \"%s\", \"threads\": %d, "
           "\"thresholds_s\": %.3f, \"ground_truth_s\": %.3f, \"total_s\": %.3f, \"kept_per_row\": %.2f, \"pairs\": [",
           n, nq, d, K, amx ? "amx-bf16" : "avx512-fp32", omp_get_max_threads(), thr_s, gt_s, now_s() - t_all,
           (double)kept / n);
    for (uint32_t t = 0; t < nks; t++) printf("%s%llu", t ? ", " : "", (unsigned long long)pairs[t]);
    printf("]}\n");
    return 0;
}
