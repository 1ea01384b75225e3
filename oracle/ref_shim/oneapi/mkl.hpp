// CPU stand-in for the two oneMKL INT8 GEMM entry points that MacraMacra/OS2-Xe's
// src/ozaki2_gpu.hpp calls (gemm_batch :1029-1033, :886-889; gemm_bias :1036-1040).
// Both compute exact int8 x int8 -> int32 products, which is all the reference relies on
// (alpha = 1, beta = 0, zero offsets). TEST INFRASTRUCTURE ONLY.
#pragma once

#include <sycl/sycl.hpp>

#include <cstdint>
#include <stdexcept>
#include <vector>

namespace oneapi {
namespace mkl {
enum class transpose { nontrans, trans, conjtrans };
enum class offset { fix, row, column };
namespace blas {
enum class compute_mode { unset, standard };
namespace column_major {
namespace detail {
// C (m x n, ldc) = op(A) op(B), op(A) is m x k, op(B) is k x n, column-major
inline void i8_gemm(transpose ta, transpose tb, int64_t m, int64_t n, int64_t k, const int8_t* a, int64_t lda,
                    const int8_t* b, int64_t ldb, int32_t* c, int64_t ldc) {
    std::vector<int8_t> at(static_cast<size_t>(m) * k);  // op(A) rows, k contiguous
    for (int64_t i = 0; i < m; ++i)
        for (int64_t p = 0; p < k; ++p)
            at[static_cast<size_t>(i) * k + p] = ta == transpose::nontrans ? a[i + p * lda] : a[p + i * lda];
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < n; ++j) {
        std::vector<int8_t> bj(static_cast<size_t>(k));
        for (int64_t p = 0; p < k; ++p) bj[p] = tb == transpose::nontrans ? b[p + j * ldb] : b[j + p * ldb];
        for (int64_t i = 0; i < m; ++i) {
            const int8_t* ar = &at[static_cast<size_t>(i) * k];
            int32_t acc = 0;
            for (int64_t p = 0; p < k; ++p) acc += static_cast<int32_t>(ar[p]) * static_cast<int32_t>(bj[p]);
            c[i + j * ldc] = acc;
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
