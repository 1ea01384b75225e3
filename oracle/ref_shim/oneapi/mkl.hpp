// CPU stand-in for the two oneMKL INT8 GEMM entry points that MacraMacra/OS2-Xe's
// src/ozaki2_gpu.hpp calls (gemm_batch :1029-1033, :886-889; gemm_bias :1036-1040).
// Both compute exact int8 x int8 -> int32 products, which is all the reference relies on
// (alpha = 1, beta = 0, zero offsets). TEST INFRASTRUCTURE ONLY.
#pragma once

#include <sycl/sycl.hpp>

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <vector>
#if defined(__x86_64__)
#include <immintrin.h>
#endif

namespace oneapi {
namespace mkl {
enum class transpose { nontrans, trans, conjtrans };
enum class offset { fix, row, column };
namespace blas {
enum class compute_mode { unset, standard };
namespace column_major {
namespace detail {
// Dot products of two rows of op(A) with two columns of op(B), all k-contiguous int8:
// out = {a0.b0, a1.b0, a0.b1, a1.b1}. AVX-512 VNNI or AVX2 where the CPU has them (sign-extension
// to int16 and pairwise multiply-add into int32 lanes: exact, |sum| < 2^31 as in the reference's
// own bound), plain loops otherwise.
#if defined(__x86_64__)
__attribute__((target("avx2"))) static inline void dot2x2_avx2(const int8_t* a0, const int8_t* a1,
                                                               const int8_t* b0, const int8_t* b1, int64_t k,
                                                               int32_t* out) {
    __m256i s00 = _mm256_setzero_si256(), s10 = s00, s01 = s00, s11 = s00;
    int64_t p = 0;
    for (; p + 16 <= k; p += 16) {
        const __m256i x0 = _mm256_cvtepi8_epi16(_mm_loadu_si128(reinterpret_cast<const __m128i*>(a0 + p)));
        const __m256i x1 = _mm256_cvtepi8_epi16(_mm_loadu_si128(reinterpret_cast<const __m128i*>(a1 + p)));
        const __m256i y0 = _mm256_cvtepi8_epi16(_mm_loadu_si128(reinterpret_cast<const __m128i*>(b0 + p)));
        const __m256i y1 = _mm256_cvtepi8_epi16(_mm_loadu_si128(reinterpret_cast<const __m128i*>(b1 + p)));
        s00 = _mm256_add_epi32(s00, _mm256_madd_epi16(x0, y0));
        s10 = _mm256_add_epi32(s10, _mm256_madd_epi16(x1, y0));
        s01 = _mm256_add_epi32(s01, _mm256_madd_epi16(x0, y1));
        s11 = _mm256_add_epi32(s11, _mm256_madd_epi16(x1, y1));
    }
    const __m256i* v[4] = {&s00, &s10, &s01, &s11};
    for (int q = 0; q < 4; ++q) {
        alignas(32) int32_t t[8];
        _mm256_store_si256(reinterpret_cast<__m256i*>(t), *v[q]);
        out[q] = t[0] + t[1] + t[2] + t[3] + t[4] + t[5] + t[6] + t[7];
    }
    for (; p < k; ++p) {
        out[0] += a0[p] * b0[p];
        out[1] += a1[p] * b0[p];
        out[2] += a0[p] * b1[p];
        out[3] += a1[p] * b1[p];
    }
}
__attribute__((target("avx512f,avx512bw,avx512vnni"))) static inline void dot2x2_vnni(
    const int8_t* a0, const int8_t* a1, const int8_t* b0, const int8_t* b1, int64_t k, int32_t* out) {
    __m512i s00 = _mm512_setzero_si512(), s10 = s00, s01 = s00, s11 = s00;
    int64_t p = 0;
    for (; p + 32 <= k; p += 32) {
        const __m512i x0 = _mm512_cvtepi8_epi16(_mm256_loadu_si256(reinterpret_cast<const __m256i*>(a0 + p)));
        const __m512i x1 = _mm512_cvtepi8_epi16(_mm256_loadu_si256(reinterpret_cast<const __m256i*>(a1 + p)));
        const __m512i y0 = _mm512_cvtepi8_epi16(_mm256_loadu_si256(reinterpret_cast<const __m256i*>(b0 + p)));
        const __m512i y1 = _mm512_cvtepi8_epi16(_mm256_loadu_si256(reinterpret_cast<const __m256i*>(b1 + p)));
        s00 = _mm512_dpwssd_epi32(s00, x0, y0);
        s10 = _mm512_dpwssd_epi32(s10, x1, y0);
        s01 = _mm512_dpwssd_epi32(s01, x0, y1);
        s11 = _mm512_dpwssd_epi32(s11, x1, y1);
    }
    out[0] = _mm512_reduce_add_epi32(s00);
    out[1] = _mm512_reduce_add_epi32(s10);
    out[2] = _mm512_reduce_add_epi32(s01);
    out[3] = _mm512_reduce_add_epi32(s11);
    for (; p < k; ++p) {
        out[0] += a0[p] * b0[p];
        out[1] += a1[p] * b0[p];
        out[2] += a0[p] * b1[p];
        out[3] += a1[p] * b1[p];
    }
}
#endif
static inline void dot2x2_plain(const int8_t* a0, const int8_t* a1, const int8_t* b0, const int8_t* b1, int64_t k,
                                int32_t* out) {
    int32_t s00 = 0, s10 = 0, s01 = 0, s11 = 0;
    for (int64_t p = 0; p < k; ++p) {
        s00 += a0[p] * b0[p];
        s10 += a1[p] * b0[p];
        s01 += a0[p] * b1[p];
        s11 += a1[p] * b1[p];
    }
    out[0] = s00, out[1] = s10, out[2] = s01, out[3] = s11;
}
// 2: AVX-512 VNNI, 1: AVX2, 0: plain loops (chosen once, from the CPU the process runs on)
static inline int simd_level() {
#if defined(__x86_64__)
    static const int lv = __builtin_cpu_supports("avx512vnni") && __builtin_cpu_supports("avx512bw")
                              ? 2
                              : (__builtin_cpu_supports("avx2") ? 1 : 0);
    return lv;
#else
    return 0;
#endif
}

// C (m x n, ldc) = op(A) op(B), op(A) is m x k, op(B) is k x n, column-major. Both operands are
// first copied k-contiguous (rows of op(A), columns of op(B), zero-padded to even counts); C is
// then computed in 64 x 64 blocks (one OpenMP task each, the two 64-row / 64-column int8 panels
// stay in the core's cache) of 2 x 2 dot products.
inline void i8_gemm(transpose ta, transpose tb, int64_t m, int64_t n, int64_t k, const int8_t* a, int64_t lda,
                    const int8_t* b, int64_t ldb, int32_t* c, int64_t ldc) {
    const int64_t m2 = m + (m & 1), n2 = n + (n & 1);
    std::vector<int8_t> at(static_cast<size_t>(m2) * k, 0), bt(static_cast<size_t>(n2) * k, 0);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; ++i)
        for (int64_t p = 0; p < k; ++p)
            at[static_cast<size_t>(i) * k + p] = ta == transpose::nontrans ? a[i + p * lda] : a[p + i * lda];
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < n; ++j)
        for (int64_t p = 0; p < k; ++p)
            bt[static_cast<size_t>(j) * k + p] = tb == transpose::nontrans ? b[p + j * ldb] : b[j + p * ldb];
    constexpr int64_t kBlk = 64;
    const int64_t bi = (m2 + kBlk - 1) / kBlk, bj = (n2 + kBlk - 1) / kBlk;
    const int simd = simd_level();
#pragma omp parallel for schedule(dynamic)
    for (int64_t blk = 0; blk < bi * bj; ++blk) {
        const int64_t i0 = (blk % bi) * kBlk, j0 = (blk / bi) * kBlk;
        const int64_t i1 = std::min(m2, i0 + kBlk), j1 = std::min(n2, j0 + kBlk);
        for (int64_t j = j0; j < j1; j += 2)
            for (int64_t i = i0; i < i1; i += 2) {
                const int8_t* a0 = &at[static_cast<size_t>(i) * k];
                const int8_t* b0 = &bt[static_cast<size_t>(j) * k];
                int32_t o[4] = {0, 0, 0, 0};
#if defined(__x86_64__)
                if (simd == 2) dot2x2_vnni(a0, a0 + k, b0, b0 + k, k, o);
                else if (simd == 1) dot2x2_avx2(a0, a0 + k, b0, b0 + k, k, o);
                else dot2x2_plain(a0, a0 + k, b0, b0 + k, k, o);
#else
                dot2x2_plain(a0, a0 + k, b0, b0 + k, k, o);
#endif
                if (i < m && j < n) c[i + j * ldc] = o[0];
                if (i + 1 < m && j < n) c[i + 1 + j * ldc] = o[1];
                if (i < m && j + 1 < n) c[i + (j + 1) * ldc] = o[2];
                if (i + 1 < m && j + 1 < n) c[i + 1 + (j + 1) * ldc] = o[3];
            }
    }
}
}  // namespace detail

inline sycl::event gemm_batch(sycl::queue&, transpose ta, transpose tb, int64_t m, int64_t n, int64_t k,
                              float alpha, const int8_t* a, int64_t lda, int64_t stride_a, const int8_t* b,
                              int64_t ldb, int64_t stride_b, float beta, int32_t* c, int64_t ldc, int64_t stride_c,
                              int64_t batch, compute_mode = compute_mode::unset,
                              const std::vector<sycl::event>& = {}) {
    if (alpha != 1.0f || beta != 0.0f) throw std::logic_error("int8 stand-in supports alpha=1, beta=0 only");
    for (int64_t q = 0; q < batch; ++q)
        detail::i8_gemm(ta, tb, m, n, k, a + q * stride_a, lda, b + q * stride_b, ldb, c + q * stride_c, ldc);
    return sycl::event{};
}

inline sycl::event gemm_bias(sycl::queue&, transpose ta, transpose tb, offset, int64_t m, int64_t n, int64_t k,
                             float alpha, const int8_t* a, int64_t lda, int8_t ao, const int8_t* b, int64_t ldb,
                             int8_t bo, float beta, int32_t* c, int64_t ldc, const int32_t* co,
                             compute_mode = compute_mode::unset, const std::vector<sycl::event>& = {}) {
    if (alpha != 1.0f || beta != 0.0f || ao != 0 || bo != 0 || co[0] != 0)
        throw std::logic_error("int8 stand-in supports plain products only");
    detail::i8_gemm(ta, tb, m, n, k, a, lda, b, ldb, c, ldc);
    return sycl::event{};
}
}  // namespace column_major
}  // namespace blas
}  // namespace mkl
}  // namespace oneapi
