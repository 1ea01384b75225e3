/*
 * oz2_oracle.h - CPU oracle for the Ozaki Scheme II FP64 GEMM emulation path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA path: only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs
 * load it. The product library (liboz2.so) never links or calls it.
 *
 * It restates, in plain C, the arithmetic of the reference header
 * src/ozaki2_gpu.hpp (MacraMacra/OS2-Xe):
 *   - modulus sets and the plan (M, tk, CRT weights)      :149-200, src/coprime_tables.hpp
 *   - exponent rule D = tk - frexp_exp(max|x|)            :360-377
 *   - exact RNE scaling to integers from the double bits  :251-289
 *   - symmetric residues in [-h, m-1-h], h = (m-1)/2      :407-455, :457-520
 *   - exact INT8 products (any exact GEMM is equivalent)  :1029-1040
 *   - CRT reconstruction + one rounding + ldexp           :526-588, :603-664
 * and of the reference test tests/test_ozaki2.cpp:
 *   - double-double dot product                           :56-84, :356-377
 *   - element-wise rigorous bound                         :155-178, :405-429
 * and the accuracy metrics of benchmarks/bench_accuracy.cpp:69-94.
 *
 * The CRT here is computed with exact multi-word integers (x = sum r_t W_t mod M,
 * symmetric representative), not with the reference's FP32 quotient estimate; the
 * two agree whenever |x| <= M/4, which the plan's tk guarantees.
 */
#ifndef OZ2_ORACLE_H
#define OZ2_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OZ2O_MAX_MODULI 24      /* the reference's range of s */
#define OZ2O_MAX_MODULI_EXT 32  /* the product's adaptive path: its own sets for s = 25..32 */
#define OZ2O_BIG_WORDS 8
#define OZ2O_NON_FINITE (-2147483647 - 1)

typedef struct {
    int s;        /* number of moduli */
    int nl;       /* 32-bit limbs needed for M */
    int tk;       /* bits per scaled element */
    double log2M;
    uint32_t m[OZ2O_MAX_MODULI_EXT];
    uint32_t y[OZ2O_MAX_MODULI_EXT];                 /* (M/m_t)^-1 mod m_t */
    uint32_t W[OZ2O_MAX_MODULI_EXT][OZ2O_BIG_WORDS]; /* (M/m_t) * y_t */
    uint32_t M[OZ2O_BIG_WORDS];
} oz2o_plan;

/* status codes shared with the product's C ABI */
#define OZ2O_OK 0
#define OZ2O_EINVAL 1
#define OZ2O_EINTERNAL 3
#define OZ2O_EOVERFLOW 5

int oz2o_moduli(int s, uint32_t* out);
int oz2o_make_plan(int s, int64_t k, oz2o_plan* p);
/* s in [2, 32]: the reference's plans up to 24, above that the product library's extended sets
 * (no counterpart in the reference; pairwise-coprime moduli <= 256 greedily from the top, tk up
 * to 124), restated so the GPU's extended path can be checked bit for bit */
int oz2o_make_plan_ext(int s, int64_t k, oz2o_plan* p);
int oz2o_precision_bits(int64_t k, int s, int* out);
int oz2o_moduli_for_bits(int64_t k, int bits);

/* exponent for one row/column from the raw bits of its max |x| */
int oz2o_exponent(uint64_t maxbits, int tk);

/* x = RNE(v * 2^e): sign and magnitude (low, high 64-bit words) */
void oz2o_scaled_int(double v, int e, int* neg, uint64_t* lo, uint64_t* hi);

/* symmetric residue of the scaled integer of v modulo m, as the stored int8 byte */
int8_t oz2o_residue(double v, int e, uint32_t m);

/* split a column-major rows x cols matrix into s planes P[t*plane + r + c*ldp];
 * per_row: exponent ex[r] per row, else ex[c] per column. */
void oz2o_split(const double* X, int64_t ldx, int64_t rows, int64_t cols, const int* ex, int per_row,
                const oz2o_plan* p, int8_t* P, int64_t ldp, int64_t plane);

/* CRT: residues r[t] (any integers congruent mod m_t) -> rounded double * 2^-shift */
double oz2o_crt(const oz2o_plan* p, const int64_t* r, int shift);

/* full emulated DGEMM on the CPU, C = alpha op(A) op(B) + beta C, ops 'N','T','C' */
/* oz2o_dgemm at s in [2, 32] through oz2o_make_plan_ext (the product's adaptive path) */
int oz2o_dgemm_ext(char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A, int64_t lda,
                   const double* B, int64_t ldb, double beta, double* C, int64_t ldc, int s);
int oz2o_dgemm(char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A, int64_t lda,
               const double* B, int64_t ldb, double beta, double* C, int64_t ldc, int s);
/* complex (interleaved re,im) ZGEMM via exact 3M; alpha, beta are [re, im] */
int oz2o_zgemm(char ta, char tb, int64_t m, int64_t n, int64_t k, const double* alpha, const double* A,
               int64_t lda, const double* B, int64_t ldb, const double* beta, double* C, int64_t ldc, int s);

/* row exponents of op(A) and column exponents of op(B) (complex: pair max of re/im) */
void oz2o_exponents(char ta, char tb, int64_t m, int64_t n, int64_t k, const double* A, int64_t lda,
                    const double* B, int64_t ldb, int tk, int cplx, int* D, int* E);

/* double-double reference: hi + lo ~= op(A) op(B) (m x n column-major, ld m) */
void oz2o_dd_gemm(char ta, char tb, int64_t m, int64_t n, int64_t k, const double* A, int64_t lda,
                  const double* B, int64_t ldb, double* hi, double* lo);
void oz2o_dd_zgemm(char ta, char tb, int64_t m, int64_t n, int64_t k, const double* A, int64_t lda,
                   const double* B, int64_t ldb, double* hi, double* lo);

/* rigorous element-wise bound of the reference test; returns max err/bound.
 * C0 is C before the call (used when alpha != 1 or beta != 0). */
double oz2o_bound_ratio(char ta, char tb, int64_t m, int64_t n, int64_t k, int s, const double* A, int64_t lda,
                        const double* B, int64_t ldb, double alpha, double beta, const double* C0,
                        const double* C, int64_t ldc, const double* hi, const double* lo);
double oz2o_zbound_ratio(char ta, char tb, int64_t m, int64_t n, int64_t k, int s, const double* A, int64_t lda,
                         const double* B, int64_t ldb, const double* alpha, const double* beta, const double* C0,
                         const double* C, int64_t ldc, const double* hi, const double* lo);

/* accuracy metrics of C (m*n contiguous values) against hi+lo:
 * out = {ulp_max, ulp_mean, cr_frac, ab_max, fro_rel}; absAB may be NULL. */
void oz2o_metrics(int64_t count, const double* C, const double* hi, const double* lo, const double* absAB,
                  double* out);

/* Ozaki Scheme I, the reference's comparison baseline (benchmarks/ozaki1_gpu.hpp): C = A B (N, N)
 * with L digits of 7 bits, tk = 7L - 2; returns OZ2O_EINVAL for L outside [2, 9] or k * 4096 >= 2^31,
 * OZ2O_EINTERNAL when memory runs out */
int oz1o_precision_bits(int L);
int oz1o_dgemm(int64_t m, int64_t n, int64_t k, const double* A, int64_t lda, const double* B, int64_t ldb,
               double* C, int64_t ldc, int L);

/* threads used by the oracle's parallel loops (1 = serial) */
void oz2o_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
