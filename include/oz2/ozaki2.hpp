// ozaki2.hpp - the oz2::Ozaki2 C++ API of MacraMacra/OS2-Xe (src/ozaki2_gpu.hpp:678-1188) over
// the C ABI of liboz2.so (oz2/oz2.h). Same member names, argument order, and exception types
// (std::invalid_argument, std::runtime_error, std::overflow_error); the SYCL queue becomes a
// CUDA stream and sycl::event dependencies become cudaEvent_t. Link with -loz2.
#pragma once

#include <cuda_runtime_api.h>

#include <complex>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "oz2/oz2.h"

namespace oz2 {

inline constexpr int kMaxModuli = 24;

enum class Trans { N, T, C };

struct StageTimes {
    double scale_ms = 0, split_ms = 0, gemm_ms = 0, crt_ms = 0;
    double total_ms() const { return scale_ms + split_ms + gemm_ms + crt_ms; }
};

struct Tuning {
    bool batched_gemm = true;
    bool pad_lda = true;
    bool pow2_tiles = true;
};

struct TileInfo {
    int64_t mb = 0, nb = 0;
    int64_t pm = 0, pn = 0;
    int64_t k_chunks = 0;
    size_t workspace_bytes = 0;
};

namespace detail {
inline void check(int status, oz2_handle h = nullptr) {
    if (status == OZ2_OK) return;
    const std::string msg = oz2_last_error(h);
    switch (status) {
        case OZ2_EINVAL: throw std::invalid_argument(msg);
        case OZ2_EOVERFLOW: throw std::overflow_error(msg);
        default: throw std::runtime_error(msg.empty() ? oz2_status_string(status) : msg);
    }
}
inline char op(Trans t) { return t == Trans::N ? 'N' : (t == Trans::T ? 'T' : 'C'); }
}  // namespace detail

class Ozaki2 {
public:
    // binds to a caller-owned stream that must outlive the object; profiling enables stage_times()
    explicit Ozaki2(cudaStream_t stream = nullptr, bool profiling = false) {
        detail::check(oz2_create(stream, &h_));
        if (profiling) detail::check(oz2_set_profiling(h_, 1), h_);
    }
    ~Ozaki2() { oz2_destroy(h_); }
    Ozaki2(const Ozaki2&) = delete;
    Ozaki2& operator=(const Ozaki2&) = delete;

    static int precision_bits(int64_t k, int num_moduli) {
        int v = 0;
        detail::check(oz2_precision_bits(k, num_moduli, &v));
        return v;
    }
    static int precision_bits_complex(int64_t k, int num_moduli) {
        int v = 0;
        detail::check(oz2_precision_bits_complex(k, num_moduli, &v));
        return v;
    }
    static int moduli_for_bits(int64_t k, int bits) {
        int v = 0;
        detail::check(oz2_moduli_for_bits(k, bits, &v));
        return v;
    }

    void set_workspace_limit(size_t bytes) { detail::check(oz2_set_workspace_limit(h_, bytes), h_); }
    void set_resident_hint(size_t bytes) { detail::check(oz2_set_resident_hint(h_, bytes), h_); }
    void release_workspace() { detail::check(oz2_release_workspace(h_), h_); }

    TileInfo last_tiling() const {
        int64_t v[6];
        detail::check(oz2_last_tiling(h_, v), h_);
        return TileInfo{v[0], v[1], v[2], v[3], v[4], static_cast<size_t>(v[5])};
    }
    void set_tuning(const Tuning& t) {
        tune_ = t;
        detail::check(oz2_set_tuning(h_, t.batched_gemm, t.pad_lda, t.pow2_tiles), h_);
    }
    const Tuning& tuning() const { return tune_; }

    StageTimes stage_times() {
        double v[4];
        detail::check(oz2_stage_times(h_, v), h_);
        return StageTimes{v[0], v[1], v[2], v[3]};
    }

    // C = alpha op(A) op(B) + beta C; device pointers, column-major; asynchronous on the stream.
    // `done` (optional) is recorded after the last kernel of the call.
    void gemm(Trans ta, Trans tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A, int64_t lda,
              const double* B, int64_t ldb, double beta, double* C, int64_t ldc, int num_moduli,
              const std::vector<cudaEvent_t>& deps = {}, cudaEvent_t done = nullptr) {
        std::vector<void*> d(deps.begin(), deps.end());
        detail::check(oz2_dgemm(h_, detail::op(ta), detail::op(tb), m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                                num_moduli, d.data(), static_cast<int>(d.size()), done),
                      h_);
    }

    void zgemm(Trans ta, Trans tb, int64_t m, int64_t n, int64_t k, std::complex<double> alpha,
               const std::complex<double>* A, int64_t lda, const std::complex<double>* B, int64_t ldb,
               std::complex<double> beta, std::complex<double>* C, int64_t ldc, int num_moduli,
               const std::vector<cudaEvent_t>& deps = {}, cudaEvent_t done = nullptr) {
        const double al[2] = {alpha.real(), alpha.imag()}, be[2] = {beta.real(), beta.imag()};
        std::vector<void*> d(deps.begin(), deps.end());
        detail::check(oz2_zgemm(h_, detail::op(ta), detail::op(tb), m, n, k, al, reinterpret_cast<const double*>(A),
                                lda, reinterpret_cast<const double*>(B), ldb, be, reinterpret_cast<double*>(C), ldc,
                                num_moduli, d.data(), static_cast<int>(d.size()), done),
                      h_);
    }

    // synchronises the stream; throws std::runtime_error if a kernel's bounded wait ran out
    void check_device_error() { detail::check(oz2_check_device_error(h_), h_); }

    oz2_handle handle() const { return h_; }

private:
    oz2_handle h_ = nullptr;
    Tuning tune_{};
};

}  // namespace oz2
