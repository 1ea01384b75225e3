/*
 * oz2_oracle.c - CPU oracle for the Ozaki Scheme II emulation path (see oz2_oracle.h).
 *
 * TEST INFRASTRUCTURE ONLY: the checker, never the thing measured or shipped.
 * Built with -ffp-contract=off so that every floating-point expression rounds
 * exactly as written: the alpha/beta updates are the reference's literal unfused
 * expressions (src/ozaki2_gpu.hpp:625, :654-660, :1066, :917-923), which the CUDA
 * kernels also evaluate operation by operation.
 */
#include "oz2_oracle.h"

#include <math.h>
#include <string.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------------------------------
 * Modulus sets. The reference lists pairwise-coprime moduli <= 256 per s
 * (src/coprime_tables.hpp:10-111, COPRIME_DATA at COPRIME_OFFSET[s]). For the s range
 * used by the path (2..24) every set is a prefix of one of three sequences.
 * ------------------------------------------------------------------------------------------ */
static const uint16_t kSeqSmall[6] = {256, 255, 253, 251, 247, 241};                       /* s = 2..6  */
static const uint16_t kSeqMid[13] = {256, 253, 251, 249, 247, 245, 241, 239, 233, 229, 227, 223, 211}; /* 7..13 */
static const uint16_t kSeqLarge[24] = {256, 253, 251, 249, 247, 241, 239, 235, 233, 229, 227, 223,
                                       217, 211, 199, 197, 193, 191, 181, 179, 173, 167, 163, 157}; /* 14..24 */

/* the product library's extended sets (s = 25..32; no counterpart in the reference) */
static const uint16_t kSeqExt[32] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193,
                                     191, 181, 179, 173, 167, 163, 157, 151, 149, 139, 137, 131, 127, 113, 109, 107};

int oz2o_moduli(int s, uint32_t* out) {
    if (s < 2 || s > OZ2O_MAX_MODULI_EXT) return OZ2O_EINVAL;
    const uint16_t* seq = s <= 6 ? kSeqSmall : (s <= 13 ? kSeqMid : (s <= OZ2O_MAX_MODULI ? kSeqLarge : kSeqExt));
    for (int t = 0; t < s; ++t) out[t] = seq[t];
    return OZ2O_OK;
}

/* ------------------------------------------------------------------------------------------
 * Fixed-width unsigned integers of OZ2O_BIG_WORDS 32-bit words (little endian).
 * ------------------------------------------------------------------------------------------ */
typedef struct { uint32_t w[OZ2O_BIG_WORDS]; } big;

static void big_zero(big* a) { memset(a, 0, sizeof *a); }
static void big_u64(big* a, uint64_t v) { big_zero(a); a->w[0] = (uint32_t)v; a->w[1] = (uint32_t)(v >> 32); }

static int big_mul_small(big* a, uint32_t f) {
    uint64_t c = 0;
    for (int i = 0; i < OZ2O_BIG_WORDS; ++i) {
        uint64_t t = (uint64_t)a->w[i] * f + c;
        a->w[i] = (uint32_t)t;
        c = t >> 32;
    }
    return c ? OZ2O_EOVERFLOW : OZ2O_OK;
}
static int big_add_small(big* a, uint32_t v) {
    uint64_t c = v;
    for (int i = 0; i < OZ2O_BIG_WORDS && c; ++i) {
        uint64_t t = (uint64_t)a->w[i] + c;
        a->w[i] = (uint32_t)t;
        c = t >> 32;
    }
    return c ? OZ2O_EOVERFLOW : OZ2O_OK;
}
static uint32_t big_divmod_small(big* a, uint32_t d) {
    uint64_t r = 0;
    for (int i = OZ2O_BIG_WORDS - 1; i >= 0; --i) {
        uint64_t cur = (r << 32) | a->w[i];
        a->w[i] = (uint32_t)(cur / d);
        r = cur % d;
    }
    return (uint32_t)r;
}
static uint32_t big_mod_small(const big* a, uint32_t d) { big t = *a; return big_divmod_small(&t, d); }
static int big_cmp(const big* a, const big* b) {
    for (int i = OZ2O_BIG_WORDS - 1; i >= 0; --i)
        if (a->w[i] != b->w[i]) return a->w[i] < b->w[i] ? -1 : 1;
    return 0;
}
static void big_sub(big* r, const big* a, const big* b) { /* r = a - b, a >= b */
    int64_t br = 0;
    for (int i = 0; i < OZ2O_BIG_WORDS; ++i) {
        int64_t t = (int64_t)a->w[i] - b->w[i] - br;
        br = t < 0;
        r->w[i] = (uint32_t)(t + (br ? ((int64_t)1 << 32) : 0));
    }
}
static int big_shl(big* a, int bits) { /* returns overflow if bits are shifted out */
    big r; big_zero(&r);
    for (int b = OZ2O_BIG_WORDS * 32 - bits; b < OZ2O_BIG_WORDS * 32; ++b)
        if (b >= 0 && ((a->w[b / 32] >> (b % 32)) & 1u)) return OZ2O_EOVERFLOW;
    for (int b = 0; b + bits < OZ2O_BIG_WORDS * 32; ++b)
        if ((a->w[b / 32] >> (b % 32)) & 1u) r.w[(b + bits) / 32] |= 1u << ((b + bits) % 32);
    *a = r;
    return OZ2O_OK;
}
static int big_top_bit(const big* a) {
    for (int i = OZ2O_BIG_WORDS - 1; i >= 0; --i)
        if (a->w[i]) return i * 32 + 31 - __builtin_clz(a->w[i]);
    return -1;
}
static int big_bit(const big* a, int i) { return i < 0 ? 0 : (int)((a->w[i / 32] >> (i % 32)) & 1u); }

/* log2 from the top three words, the estimate the reference's tk search starts from
 * (src/ozaki2_gpu.hpp:127-135) */
static double big_log2(const big* a) {
    int top = OZ2O_BIG_WORDS - 1;
    while (top > 0 && a->w[top] == 0) --top;
    double v = 0;
    int lo = top - 2 > 0 ? top - 2 : 0;
    for (int i = top; i >= lo; --i) v = v * 4294967296.0 + a->w[i];
    return log2(v) + 32.0 * (top - 2 > 0 ? top - 2 : 0);
}

static int64_t mod_inverse(int64_t a, int64_t m) {
    int64_t t = 0, nt = 1, r = m, nr = ((a % m) + m) % m;
    while (nr) {
        int64_t q = r / nr, tmp;
        tmp = t - q * nt; t = nt; nt = tmp;
        tmp = r - q * nr; r = nr; nr = tmp;
    }
    if (r != 1) return -1;
    return (t % m + m) % m;
}

/* plan: ref src/ozaki2_gpu.hpp:159-200 (s <= 24); the same rule with tk capped at 124 for the
 * extended sets */
int oz2o_make_plan(int s, int64_t k, oz2o_plan* p) {
    if (s > OZ2O_MAX_MODULI) return OZ2O_EINVAL;
    return oz2o_make_plan_ext(s, k, p);
}

int oz2o_make_plan_ext(int s, int64_t k, oz2o_plan* p) {
    if (s < 2 || s > OZ2O_MAX_MODULI_EXT || k < 1) return OZ2O_EINVAL;
    memset(p, 0, sizeof *p);
    p->s = s;
    oz2o_moduli(s, p->m);
    big M; big_u64(&M, 1);
    for (int t = 0; t < s; ++t)
        if (big_mul_small(&M, p->m[t])) return OZ2O_EOVERFLOW;
    p->log2M = big_log2(&M);
    p->nl = (int)floor(p->log2M / 32.0) + 1;
    if (p->nl < 2) p->nl = 2;
    int tk = (int)floor((p->log2M - 2.0 - log2((double)k)) / 2.0);
    const int cap = s <= OZ2O_MAX_MODULI ? 100 : 124;
    if (tk > cap) tk = cap;
    for (;; --tk) {
        if (tk < 1) return OZ2O_EINVAL;
        big lhs; big_u64(&lhs, (uint64_t)k);
        if (big_shl(&lhs, 2 * tk + 2)) continue;
        if (big_cmp(&lhs, &M) <= 0) break;
    }
    p->tk = tk;
    for (int t = 0; t < s; ++t) {
        big Mt = M;
        if (big_divmod_small(&Mt, p->m[t]) != 0) return OZ2O_EINVAL;
        int64_t y = mod_inverse(big_mod_small(&Mt, p->m[t]), p->m[t]);
        if (y < 0) return OZ2O_EINVAL;
        if (big_mul_small(&Mt, (uint32_t)y)) return OZ2O_EOVERFLOW;
        memcpy(p->W[t], Mt.w, sizeof Mt.w);
        p->y[t] = (uint32_t)y;
    }
    memcpy(p->M, M.w, sizeof M.w);
    return OZ2O_OK;
}

int oz2o_precision_bits(int64_t k, int s, int* out) {
    oz2o_plan p;
    int st = oz2o_make_plan(s, k, &p);
    if (st == OZ2O_OK) *out = p.tk;
    return st;
}

/* ref src/ozaki2_gpu.hpp:693-700 */
int oz2o_moduli_for_bits(int64_t k, int bits) {
    for (int s = 2; s <= OZ2O_MAX_MODULI; ++s) {
        oz2o_plan p;
        if (oz2o_make_plan(s, k, &p) == OZ2O_OK && p.tk >= bits) return s;
    }
    return OZ2O_MAX_MODULI;
}

/* ref src/ozaki2_gpu.hpp:364-375: D = tk - e where max = f 2^e, f in [0.5, 1) */
int oz2o_exponent(uint64_t maxbits, int tk) {
    if (maxbits >= 0x7FF0000000000000ull) return OZ2O_NON_FINITE;
    if (maxbits == 0) return 0;
    double v;
    memcpy(&v, &maxbits, 8);
    int e2;
    frexp(v, &e2);
    return tk - e2;
}

/* x = RNE(v 2^e) from the bits of v (ref src/ozaki2_gpu.hpp:251-289). |v 2^e| <= 2^124 here. */
void oz2o_scaled_int(double v, int e, int* neg, uint64_t* lo, uint64_t* hi) {
    uint64_t bits;
    memcpy(&bits, &v, 8);
    *neg = (int)(bits >> 63);
    const int be = (int)((bits >> 52) & 0x7FF);
    uint64_t mant = bits & 0xFFFFFFFFFFFFFull;
    if (be) mant |= 0x10000000000000ull;
    u128 x = 0;
    if (mant != 0 && e != OZ2O_NON_FINITE) {
        const int sh = (be ? be : 1) - 1075 + e;
        if (sh >= 0) {
            x = (u128)mant << sh;
        } else if (sh >= -54) {
            const int rs = -sh;
            const uint64_t q = mant >> rs;
            const uint64_t rem = mant & ((1ull << rs) - 1);
            const uint64_t half = 1ull << (rs - 1);
            x = q + ((rem > half || (rem == half && (q & 1))) ? 1 : 0);
        }
    }
    *lo = (uint64_t)x;
    *hi = (uint64_t)(x >> 64);
}

static int sym_residue_mag(int neg, uint64_t lo, uint64_t hi, uint32_t m) {
    const u128 x = ((u128)hi << 64) | lo;
    int r = (int)(x % m);
    if (neg) r = (int)((m - (uint32_t)r) % m);
    const int h = (int)(m - 1) / 2;
    if (r > (int)m - 1 - h) r -= (int)m;
    return r; /* in [-h, m-1-h]; 128 for m = 256 is stored as the byte 0x80 */
}

int8_t oz2o_residue(double v, int e, uint32_t m) {
    int neg;
    uint64_t lo, hi;
    oz2o_scaled_int(v, e, &neg, &lo, &hi);
    return (int8_t)(uint8_t)(sym_residue_mag(neg, lo, hi, m) & 0xFF);
}

/* ref src/ozaki2_gpu.hpp:407-455 (reference plane layout P[t*plane + r + c*ldp]) */
void oz2o_split(const double* X, int64_t ldx, int64_t rows, int64_t cols, const int* ex, int per_row,
                const oz2o_plan* p, int8_t* P, int64_t ldp, int64_t plane) {
    for (int64_t c = 0; c < cols; ++c)
        for (int64_t r = 0; r < rows; ++r) {
            const int e = per_row ? ex[r] : ex[c];
            const double v = e == OZ2O_NON_FINITE ? 0.0 : X[r + c * ldx];
            int neg;
            uint64_t lo, hi;
            oz2o_scaled_int(v, e, &neg, &lo, &hi);
            for (int t = 0; t < p->s; ++t)
                P[t * plane + r + c * ldp] = (int8_t)(uint8_t)(sym_residue_mag(neg, lo, hi, p->m[t]) & 0xFF);
        }
}

/* ------------------------------------------------------------------------------------------
 * CRT: mixed-radix (Garner) digits -> exact integer in [0, M) -> symmetric representative ->
 * one round-to-nearest-even to 53 bits -> ldexp by -shift. The reference reaches the same
 * integer through an FP32 quotient estimate (src/ozaki2_gpu.hpp:526-588); the rounding and
 * the final scaling follow :569-587.
 * ------------------------------------------------------------------------------------------ */
double oz2o_crt(const oz2o_plan* p, const int64_t* r, int shift) {
    const int s = p->s;
    int64_t a[OZ2O_MAX_MODULI_EXT];
    for (int i = 0; i < s; ++i) {
        const int64_t mi = p->m[i];
        int64_t v = ((r[i] % mi) + mi) % mi;
        for (int j = 0; j < i; ++j) {
            const int64_t inv = mod_inverse((int64_t)p->m[j] % mi, mi);
            v = ((v - a[j]) % mi + mi) % mi;
            v = (v * inv) % mi;
        }
        a[i] = v;
    }
    big x; big_zero(&x);
    for (int i = s - 1; i >= 0; --i) {
        if (i != s - 1) big_mul_small(&x, p->m[i]);
        big_add_small(&x, (uint32_t)a[i]);
    }
    big M;
    memcpy(M.w, p->M, sizeof M.w);
    big x2 = x;
    big_shl(&x2, 1);
    int neg = 0;
    if (big_cmp(&x2, &M) > 0) { /* x > M/2: negative representative */
        big t;
        big_sub(&t, &M, &x);
        x = t;
        neg = 1;
    }
    const int top = big_top_bit(&x);
    if (top < 0) return 0.0;
    uint64_t m53 = 0;
    int e = 0;
    if (top < 53) {
        for (int i = top; i >= 0; --i) m53 = (m53 << 1) | (uint64_t)big_bit(&x, i);
    } else {
        for (int i = top; i > top - 53; --i) m53 = (m53 << 1) | (uint64_t)big_bit(&x, i);
        const int rb = top - 53;
        const int round = big_bit(&x, rb);
        int sticky = 0;
        for (int i = rb - 1; i >= 0 && !sticky; --i) sticky |= big_bit(&x, i);
        if (round && (sticky || (m53 & 1))) ++m53;
        e = top - 52;
    }
    const double v = ldexp(ldexp((double)m53, e), -shift);
    return neg ? -v : v;
}

/* ------------------------------------------------------------------------------------------
 * Full CPU emulation (ref src/ozaki2_gpu.hpp:739-760 gemm, :935-1054 run, :1056-1070 scale_c,
 * :764-786 zgemm, :791-905 run_z, :907-929 scale_cz)
 * ------------------------------------------------------------------------------------------ */
static int is_n(char t) { return t == 'N' || t == 'n'; }
static int is_c(char t) { return t == 'C' || t == 'c'; }

static int check_args(char ta, char tb, int64_t m, int64_t n, int64_t k, int64_t lda, int64_t ldb, int64_t ldc) {
    if (m < 0 || n < 0 || k < 0) return OZ2O_EINVAL;
    const int64_t la = is_n(ta) ? m : k, lb = is_n(tb) ? k : n;
    if (lda < (la > 1 ? la : 1) || ldb < (lb > 1 ? lb : 1) || ldc < (m > 1 ? m : 1)) return OZ2O_EINVAL;
    return OZ2O_OK;
}

static uint64_t absbits(double v) {
    uint64_t b;
    memcpy(&b, &v, 8);
    return b & 0x7FFFFFFFFFFFFFFFull;
}

void oz2o_exponents(char ta, char tb, int64_t m, int64_t n, int64_t k, const double* A, int64_t lda,
                    const double* B, int64_t ldb, int tk, int cplx, int* D, int* E) {
    const int w = cplx ? 2 : 1;
    for (int64_t i = 0; i < m; ++i) {
        uint64_t mx = 0;
        for (int64_t p = 0; p < k; ++p) {
            const int64_t idx = is_n(ta) ? i + p * lda : p + i * lda;
            for (int c = 0; c < w; ++c) {
                const uint64_t b = absbits(A[w * idx + c]);
                if (b > mx) mx = b;
            }
        }
        D[i] = oz2o_exponent(mx, tk);
    }
    for (int64_t j = 0; j < n; ++j) {
        uint64_t mx = 0;
        for (int64_t p = 0; p < k; ++p) {
            const int64_t idx = is_n(tb) ? p + j * ldb : j + p * ldb;
            for (int c = 0; c < w; ++c) {
                const uint64_t b = absbits(B[w * idx + c]);
                if (b > mx) mx = b;
            }
        }
        E[j] = oz2o_exponent(mx, tk);
    }
}

/* exact dot product of two int8 rows */
static int64_t dot_i8(const int8_t* a, const int8_t* b, int64_t k) {
    int64_t acc = 0;
    for (int64_t p0 = 0; p0 < k; p0 += 65536) {
        const int64_t p1 = p0 + 65536 < k ? p0 + 65536 : k;
        int32_t part = 0;
        for (int64_t p = p0; p < p1; ++p) part += (int32_t)a[p] * (int32_t)b[p];
        acc += part;
    }
    return acc;
}

static double nan_value(void) { return __builtin_nan(""); }

static int dgemm_impl(char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A, int64_t lda,
                      const double* B, int64_t ldb, double beta, double* C, int64_t ldc, int s, int ext);

int oz2o_dgemm(char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A, int64_t lda,
               const double* B, int64_t ldb, double beta, double* C, int64_t ldc, int s) {
    return dgemm_impl(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s, 0);
}

int oz2o_dgemm_ext(char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A, int64_t lda,
                   const double* B, int64_t ldb, double beta, double* C, int64_t ldc, int s) {
    return dgemm_impl(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s, 1);
}

static int dgemm_impl(char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A, int64_t lda,
                      const double* B, int64_t ldb, double beta, double* C, int64_t ldc, int s, int ext) {
    if (check_args(ta, tb, m, n, k, lda, ldb, ldc)) return OZ2O_EINVAL;
    if (m == 0 || n == 0) return OZ2O_OK;
    if (k == 0 || alpha == 0.0) {
        for (int64_t j = 0; j < n; ++j)
            for (int64_t i = 0; i < m; ++i) C[i + j * ldc] = beta == 0.0 ? 0.0 : beta * C[i + j * ldc];
        return OZ2O_OK;
    }
    oz2o_plan p;
    int st = ext ? oz2o_make_plan_ext(s, k, &p) : oz2o_make_plan(s, k, &p);
    if (st) return st;
    int* D = (int*)malloc(sizeof(int) * (size_t)m);
    int* E = (int*)malloc(sizeof(int) * (size_t)n);
    int8_t* Ar = (int8_t*)malloc((size_t)s * m * k); /* [t][i][p] */
    int8_t* Br = (int8_t*)malloc((size_t)s * n * k); /* [t][j][p] */
    oz2o_exponents(ta, tb, m, n, k, A, lda, B, ldb, p.tk, 0, D, E);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; ++i)
        for (int64_t q = 0; q < k; ++q) {
            const double v = A[is_n(ta) ? i + q * lda : q + i * lda];
            int neg;
            uint64_t lo, hi;
            oz2o_scaled_int(D[i] == OZ2O_NON_FINITE ? 0.0 : v, D[i], &neg, &lo, &hi);
            for (int t = 0; t < s; ++t)
                Ar[((size_t)t * m + i) * k + q] = (int8_t)(uint8_t)(sym_residue_mag(neg, lo, hi, p.m[t]) & 0xFF);
        }
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < n; ++j)
        for (int64_t q = 0; q < k; ++q) {
            const double v = B[is_n(tb) ? q + j * ldb : j + q * ldb];
            int neg;
            uint64_t lo, hi;
            oz2o_scaled_int(E[j] == OZ2O_NON_FINITE ? 0.0 : v, E[j], &neg, &lo, &hi);
            for (int t = 0; t < s; ++t)
                Br[((size_t)t * n + j) * k + q] = (int8_t)(uint8_t)(sym_residue_mag(neg, lo, hi, p.m[t]) & 0xFF);
        }
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t j = 0; j < n; ++j)
        for (int64_t i = 0; i < m; ++i) {
            int64_t r[OZ2O_MAX_MODULI_EXT];
            for (int t = 0; t < s; ++t)
                r[t] = dot_i8(Ar + ((size_t)t * m + i) * k, Br + ((size_t)t * n + j) * k, k);
            double v = oz2o_crt(&p, r, D[i] + E[j]);
            if (D[i] == OZ2O_NON_FINITE || E[j] == OZ2O_NON_FINITE) v = nan_value();
            double* cp = C + i + j * ldc;
            *cp = beta == 0.0 ? alpha * v : alpha * v + beta * *cp;
        }
    free(D); free(E); free(Ar); free(Br);
    return OZ2O_OK;
}

int oz2o_zgemm(char ta, char tb, int64_t m, int64_t n, int64_t k, const double* alpha, const double* A,
               int64_t lda, const double* B, int64_t ldb, const double* beta, double* C, int64_t ldc, int s) {
    if (check_args(ta, tb, m, n, k, lda, ldb, ldc)) return OZ2O_EINVAL;
    if (m == 0 || n == 0) return OZ2O_OK;
    const double ar = alpha[0], ai = alpha[1], br = beta[0], bi = beta[1];
    if (k == 0 || (ar == 0.0 && ai == 0.0)) {
        for (int64_t j = 0; j < n; ++j)
            for (int64_t i = 0; i < m; ++i) {
                double* cp = C + 2 * (i + j * ldc);
                if (br == 0.0 && bi == 0.0) {
                    cp[0] = 0.0;
                    cp[1] = 0.0;
                } else {
                    const double r = cp[0], im = cp[1];
                    cp[0] = br * r - bi * im;
                    cp[1] = br * im + bi * r;
                }
            }
        return OZ2O_OK;
    }
    oz2o_plan p;
    int st = oz2o_make_plan(s, 2 * k, &p);
    if (st) return st;
    int* D = (int*)malloc(sizeof(int) * (size_t)m);
    int* E = (int*)malloc(sizeof(int) * (size_t)n);
    const size_t gA = (size_t)s * m * k, gB = (size_t)s * n * k;
    int8_t* Ar = (int8_t*)malloc(3 * gA); /* [g][t][i][p], g = re, im, re+im */
    int8_t* Br = (int8_t*)malloc(3 * gB);
    oz2o_exponents(ta, tb, m, n, k, A, lda, B, ldb, p.tk, 1, D, E);
    for (int side = 0; side < 2; ++side) {
        const int64_t rows = side ? n : m;
        const char op = side ? tb : ta;
        const double* X = side ? B : A;
        const int64_t ldx = side ? ldb : lda;
        const int* ex = side ? E : D;
        int8_t* R = side ? Br : Ar;
        const size_t g = side ? gB : gA;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < rows; ++i)
            for (int64_t q = 0; q < k; ++q) {
                int64_t idx;
                if (side) idx = is_n(op) ? q + i * ldx : i + q * ldx;
                else idx = is_n(op) ? i + q * ldx : q + i * ldx;
                double v[2] = {X[2 * idx], X[2 * idx + 1]};
                if (ex[i] == OZ2O_NON_FINITE) v[0] = v[1] = 0.0;
                if (is_c(op)) v[1] = -v[1]; /* residues of -x are the negated residues */
                int neg[2];
                uint64_t lo[2], hi[2];
                for (int c = 0; c < 2; ++c) oz2o_scaled_int(v[c], ex[i], &neg[c], &lo[c], &hi[c]);
                for (int t = 0; t < s; ++t) {
                    const int mm = (int)p.m[t], h = (mm - 1) / 2;
                    const int s0 = sym_residue_mag(neg[0], lo[0], hi[0], p.m[t]);
                    const int s1 = sym_residue_mag(neg[1], lo[1], hi[1], p.m[t]);
                    int ss = s0 + s1;
                    if (ss > mm - 1 - h) ss -= mm;
                    if (ss < -h) ss += mm;
                    const size_t o = ((size_t)t * rows + i) * k + q;
                    R[o] = (int8_t)(uint8_t)(s0 & 0xFF);
                    R[g + o] = (int8_t)(uint8_t)(s1 & 0xFF);
                    R[2 * g + o] = (int8_t)(uint8_t)(ss & 0xFF);
                }
            }
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t j = 0; j < n; ++j)
        for (int64_t i = 0; i < m; ++i) {
            int64_t rre[OZ2O_MAX_MODULI], rim[OZ2O_MAX_MODULI];
            for (int t = 0; t < s; ++t) {
                const size_t oa = ((size_t)t * m + i) * k, ob = ((size_t)t * n + j) * k;
                const int64_t p0 = dot_i8(Ar + oa, Br + ob, k);
                const int64_t p1 = dot_i8(Ar + gA + oa, Br + gB + ob, k);
                const int64_t p2 = dot_i8(Ar + 2 * gA + oa, Br + 2 * gB + ob, k);
                rre[t] = p0 - p1;
                rim[t] = p2 - p0 - p1;
            }
            double vr = oz2o_crt(&p, rre, D[i] + E[j]), vi = oz2o_crt(&p, rim, D[i] + E[j]);
            if (D[i] == OZ2O_NON_FINITE || E[j] == OZ2O_NON_FINITE) vr = vi = nan_value();
            double* cp = C + 2 * (i + j * ldc);
            double orr = ar * vr - ai * vi, oi = ar * vi + ai * vr;
            if (br != 0.0 || bi != 0.0) {
                const double cr = cp[0], ci = cp[1];
                orr += br * cr - bi * ci;
                oi += br * ci + bi * cr;
            }
            cp[0] = orr;
            cp[1] = oi;
        }
    free(D); free(E); free(Ar); free(Br);
    return OZ2O_OK;
}

/* ------------------------------------------------------------------------------------------
 * Double-double reference (ref tests/test_ozaki2.cpp:56-84, :356-377)
 * ------------------------------------------------------------------------------------------ */
static void dd_add_prod(double* sh, double* sl, double a, double b) {
    const double ph = a * b;
    const double pl = fma(a, b, -ph);
    const double s = *sh + ph;
    const double bb = s - *sh;
    const double e = (*sh - (s - bb)) + (ph - bb);
    const double t = e + *sl + pl;
    *sh = s + t;
    *sl = t - (*sh - s);
}

void oz2o_dd_gemm(char ta, char tb, int64_t m, int64_t n, int64_t k, const double* A, int64_t lda,
                  const double* B, int64_t ldb, double* hi, double* lo) {
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < n; ++j)
        for (int64_t i = 0; i < m; ++i) {
            double sh = 0, sl = 0;
            for (int64_t p = 0; p < k; ++p) {
                const double a = is_n(ta) ? A[i + p * lda] : A[p + i * lda];
                const double b = is_n(tb) ? B[p + j * ldb] : B[j + p * ldb];
                dd_add_prod(&sh, &sl, a, b);
            }
            hi[i + j * m] = sh;
            lo[i + j * m] = sl;
        }
}

void oz2o_dd_zgemm(char ta, char tb, int64_t m, int64_t n, int64_t k, const double* A, int64_t lda,
                   const double* B, int64_t ldb, double* hi, double* lo) {
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < n; ++j)
        for (int64_t i = 0; i < m; ++i) {
            double h[2] = {0, 0}, l[2] = {0, 0};
            for (int64_t p = 0; p < k; ++p) {
                const int64_t ia = is_n(ta) ? i + p * lda : p + i * lda;
                const int64_t ib = is_n(tb) ? p + j * ldb : j + p * ldb;
                const double xr = A[2 * ia], xi = is_c(ta) ? -A[2 * ia + 1] : A[2 * ia + 1];
                const double yr = B[2 * ib], yi = is_c(tb) ? -B[2 * ib + 1] : B[2 * ib + 1];
                dd_add_prod(&h[0], &l[0], xr, yr);
                dd_add_prod(&h[0], &l[0], -xi, yi);
                dd_add_prod(&h[1], &l[1], xr, yi);
                dd_add_prod(&h[1], &l[1], xi, yr);
            }
            const int64_t o = 2 * (i + j * m);
            hi[o] = h[0]; hi[o + 1] = h[1];
            lo[o] = l[0]; lo[o + 1] = l[1];
        }
}

/* ------------------------------------------------------------------------------------------
 * Rigorous bound (ref tests/test_ozaki2.cpp:128-178 real, :390-429 complex)
 * ------------------------------------------------------------------------------------------ */
static int frexp_exp(double v) { int e; frexp(v, &e); return e; }

double oz2o_bound_ratio(char ta, char tb, int64_t m, int64_t n, int64_t k, int s, const double* A, int64_t lda,
                        const double* B, int64_t ldb, double alpha, double beta, const double* C0,
                        const double* C, int64_t ldc, const double* hi, const double* lo) {
    int tk;
    if (oz2o_precision_bits(k, s, &tk)) return INFINITY;
    int* D = (int*)malloc(sizeof(int) * (size_t)m);
    int* E = (int*)malloc(sizeof(int) * (size_t)n);
    double* sa = (double*)calloc((size_t)m, sizeof(double));
    double* sb = (double*)calloc((size_t)n, sizeof(double));
    for (int64_t i = 0; i < m; ++i) {
        double mx = 0;
        for (int64_t p = 0; p < k; ++p) {
            const double v = fabs(is_n(ta) ? A[i + p * lda] : A[p + i * lda]);
            if (v > mx) mx = v;
            sa[i] += v;
        }
        D[i] = mx == 0 ? 0 : tk - frexp_exp(mx);
    }
    for (int64_t j = 0; j < n; ++j) {
        double mx = 0;
        for (int64_t p = 0; p < k; ++p) {
            const double v = fabs(is_n(tb) ? B[p + j * ldb] : B[j + p * ldb]);
            if (v > mx) mx = v;
            sb[j] += v;
        }
        E[j] = mx == 0 ? 0 : tk - frexp_exp(mx);
    }
    const double u = ldexp(1.0, -53);
    double worst = 0;
    for (int64_t j = 0; j < n; ++j)
        for (int64_t i = 0; i < m; ++i) {
            const double got = C[i + j * ldc], c0 = C0 ? C0[i + j * ldc] : 0.0;
            const double rh = hi[i + j * m], rl = lo[i + j * m];
            const double tb_err = 0.5 * ldexp(sb[j], -D[i]) + 0.5 * ldexp(sa[i], -E[j]) +
                                  0.25 * (double)k * ldexp(1.0, -D[i] - E[j]);
            double err, bound;
            if (alpha == 1.0 && beta == 0.0) {
                err = fabs((got - rh) - rl);
                bound = tb_err * (1 + 2 * u) + u * fabs(got) + 1e-300;
            } else {
                const double ref = alpha * (rh + rl) + beta * c0;
                err = fabs(got - ref);
                bound = fabs(alpha) * tb_err * (1 + 4 * u) + 4 * u * (fabs(alpha * rh) + fabs(beta * c0)) + 1e-300;
            }
            const double q = err / bound;
            if (!(q <= worst)) worst = q; /* NaN propagates as a failure */
        }
    free(D); free(E); free(sa); free(sb);
    return worst;
}

double oz2o_zbound_ratio(char ta, char tb, int64_t m, int64_t n, int64_t k, int s, const double* A, int64_t lda,
                         const double* B, int64_t ldb, const double* alpha, const double* beta, const double* C0,
                         const double* C, int64_t ldc, const double* hi, const double* lo) {
    int tk;
    if (oz2o_precision_bits(2 * k, s, &tk)) return INFINITY;
    int* D = (int*)malloc(sizeof(int) * (size_t)m);
    int* E = (int*)malloc(sizeof(int) * (size_t)n);
    double* sa = (double*)calloc((size_t)m, sizeof(double));
    double* sb = (double*)calloc((size_t)n, sizeof(double));
    for (int64_t i = 0; i < m; ++i) {
        double mx = 0;
        for (int64_t p = 0; p < k; ++p) {
            const int64_t ia = is_n(ta) ? i + p * lda : p + i * lda;
            const double r = fabs(A[2 * ia]), im = fabs(A[2 * ia + 1]);
            if (r > mx) mx = r;
            if (im > mx) mx = im;
            sa[i] += r + im;
        }
        D[i] = mx == 0 ? 0 : tk - frexp_exp(mx);
    }
    for (int64_t j = 0; j < n; ++j) {
        double mx = 0;
        for (int64_t p = 0; p < k; ++p) {
            const int64_t ib = is_n(tb) ? p + j * ldb : j + p * ldb;
            const double r = fabs(B[2 * ib]), im = fabs(B[2 * ib + 1]);
            if (r > mx) mx = r;
            if (im > mx) mx = im;
            sb[j] += r + im;
        }
        E[j] = mx == 0 ? 0 : tk - frexp_exp(mx);
    }
    const double u = ldexp(1.0, -53);
    const int plain = alpha[0] == 1.0 && alpha[1] == 0.0 && beta[0] == 0.0 && beta[1] == 0.0;
    const double aabs = hypot(alpha[0], alpha[1]);
    double worst = 0;
    for (int64_t j = 0; j < n; ++j)
        for (int64_t i = 0; i < m; ++i) {
            const int64_t o = 2 * (i + j * m), oc = 2 * (i + j * ldc);
            const double tb_err = 0.5 * ldexp(sb[j], -D[i]) + 0.5 * ldexp(sa[i], -E[j]) +
                                  0.5 * (double)k * ldexp(1.0, -D[i] - E[j]);
            const double c0r = C0 ? C0[oc] : 0.0, c0i = C0 ? C0[oc + 1] : 0.0;
            const double xr = hi[o] + lo[o], xi = hi[o + 1] + lo[o + 1];
            const double exr = alpha[0] * xr - alpha[1] * xi + (beta[0] * c0r - beta[1] * c0i);
            const double exi = alpha[0] * xi + alpha[1] * xr + (beta[0] * c0i + beta[1] * c0r);
            const double bc = hypot(beta[0] * c0r - beta[1] * c0i, beta[0] * c0i + beta[1] * c0r);
            for (int c = 0; c < 2; ++c) {
                const double g = C[oc + c];
                double err, bound;
                if (plain) {
                    err = fabs((g - hi[o + c]) - lo[o + c]);
                    bound = tb_err * (1 + 4 * u) + u * fabs(g) + 1e-300;
                } else {
                    err = fabs(g - (c ? exi : exr));
                    bound = aabs * tb_err * 2 * (1 + 8 * u) +
                            8 * u * (aabs * (fabs(hi[o]) + fabs(hi[o + 1])) + bc) + 1e-300;
                }
                const double q = err / bound;
                if (!(q <= worst)) worst = q;
            }
        }
    free(D); free(E); free(sa); free(sb);
    return worst;
}

/* ref benchmarks/bench_accuracy.cpp:69-94 */
void oz2o_metrics(int64_t count, const double* C, const double* hi, const double* lo, const double* absAB,
                  double* out) {
    double ulp_max = 0, s_ulp = 0, s_d2 = 0, s_r2 = 0, ab_max = 0;
    int64_t cr = 0;
    for (int64_t i = 0; i < count; ++i) {
        const double ref_rn = hi[i] + lo[i];
        const double err = fabs((C[i] - hi[i]) - lo[i]);
        const double ulp = hi[i] == 0 ? 4.9406564584124654e-324 : nextafter(fabs(hi[i]), INFINITY) - fabs(hi[i]);
        const double eu = err / ulp;
        if (eu > ulp_max) ulp_max = eu;
        s_ulp += eu;
        if (C[i] == ref_rn) ++cr;
        if (absAB && absAB[i] > 0 && err / absAB[i] > ab_max) ab_max = err / absAB[i];
        s_d2 += err * err;
        s_r2 += hi[i] * hi[i];
    }
    out[0] = ulp_max;
    out[1] = count ? s_ulp / (double)count : 0;
    out[2] = count ? (double)cr / (double)count : 1;
    out[3] = ab_max;
    out[4] = s_r2 > 0 ? sqrt(s_d2 / s_r2) : 0;
}

void oz2o_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : 1);
#else
    (void)n;
#endif
}

/* ---- Ozaki Scheme I, the reference's comparison baseline (benchmarks/ozaki1_gpu.hpp:10-155).
 * tk = 7L - 2 bits per element with the Ozaki-II exponent rule and RNE scaling (:116-131); each
 * scaled integer as L balanced base-128 digits, most significant first (:31-40); the digit
 * products of the first L anti-diagonals summed exactly (:139-143); Horner over the diagonals in
 * double-double, then one ldexp by 7(L - 1) - D_i - E_j, NaN for non-finite rows / columns
 * (:50-75). C = A B for column-major A (m x k), B (k x n). */
int oz1o_precision_bits(int L) { return 7 * L - 2; }

int oz1o_dgemm(int64_t m, int64_t n, int64_t k, const double* A, int64_t lda, const double* B, int64_t ldb,
               double* C, int64_t ldc, int L) {
    if (L < 2 || L > 9) return OZ2O_EINVAL;
    if (k * 4096 >= ((int64_t)1 << 31)) return OZ2O_EINVAL;
    if (m <= 0 || n <= 0) return OZ2O_OK;
    const int tk = oz1o_precision_bits(L);
    const size_t kk = (size_t)(k > 0 ? k : 1);
    int* D = (int*)malloc(sizeof(int) * (size_t)m);
    int* E = (int*)malloc(sizeof(int) * (size_t)n);
    int8_t* Ad = (int8_t*)malloc((size_t)L * (size_t)m * kk);  /* [digit][i][p] */
    int8_t* Bd = (int8_t*)malloc((size_t)L * (size_t)n * kk);  /* [digit][j][p] */
    if (!D || !E || !Ad || !Bd) {
        free(D); free(E); free(Ad); free(Bd);
        return OZ2O_EINTERNAL;
    }
    oz2o_exponents('N', 'N', m, n, k, A, lda, B, ldb, tk, 0, D, E);
    for (int side = 0; side < 2; ++side) {
        const int64_t rows = side ? n : m;
        int8_t* dst = side ? Bd : Ad;
        for (int64_t r = 0; r < rows; ++r) {
            const int ee = side ? E[r] : D[r];
            for (int64_t p = 0; p < k; ++p) {
                const double v = ee == OZ2O_NON_FINITE ? 0.0 : (side ? B[p + r * ldb] : A[r + p * lda]);
                int neg;
                uint64_t lo, hi;
                oz2o_scaled_int(v, ee, &neg, &lo, &hi);
                int64_t x = neg ? -(int64_t)lo : (int64_t)lo;
                for (int i = L - 1; i >= 0; --i) {
                    const int64_t dgt = ((x + 64) & 127) - 64;
                    x = (x - dgt) >> 7;
                    dst[((size_t)i * (size_t)rows + (size_t)r) * kk + (size_t)p] = (int8_t)dgt;
                }
            }
        }
    }
#pragma omp parallel for schedule(dynamic)
    for (int64_t j = 0; j < n; ++j)
        for (int64_t i = 0; i < m; ++i) {
            double hi = 0.0, lo = 0.0;
            for (int d = 0; d < L; ++d) {
                int64_t S = 0;
                for (int a = 0; a <= d; ++a)
                    S += dot_i8(Ad + ((size_t)a * (size_t)m + (size_t)i) * kk,
                                Bd + ((size_t)(d - a) * (size_t)n + (size_t)j) * kk, k);
                if (d > 0) {
                    hi *= 128.0;
                    lo *= 128.0;
                }
                const double sd = (double)S;
                const double s = hi + sd, bb = s - hi;
                const double err = (hi - (s - bb)) + (sd - bb) + lo;
                hi = s + err;
                lo = err - (hi - s);
            }
            double v = ldexp(hi + lo, 7 * (L - 1) - D[i] - E[j]);
            if (D[i] == OZ2O_NON_FINITE || E[j] == OZ2O_NON_FINITE) v = nan_value();
            C[i + j * ldc] = v;
        }
    free(D); free(E); free(Ad); free(Bd);
    return OZ2O_OK;
}
