// ozaki2.hpp - the oz2::Ozaki2 C++ API of MacraMacra/OS2-Xe (src/ozaki2_gpu.hpp:678-1188) over
// the C ABI of liboz2.so (oz2/oz2.h). Same member names, argument order, and exception types
// (std::invalid_argument, std::runtime_error, std::overflow_error); the SYCL queue becomes a
// CUDA stream and sycl::event dependencies become cudaEvent_t. Link with -loz2.
#pragma once

#include <cuda_runtime_api.h>

#include <array>
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

// one problem of a grouped or adaptive call (no counterpart in the reference): the arguments of
// gemm(); num_moduli is ignored by the adaptive modes other than Fixed, and in gemm_grouped
// OZ2_S_ADAPTIVE (-1) gives the problem the adaptive s per tile
struct Problem {
    Trans ta = Trans::N, tb = Trans::N;
    int64_t m = 0, n = 0, k = 0;
    double alpha = 1.0;
    const double* A = nullptr;
    int64_t lda = 1;
    const double* B = nullptr;
    int64_t ldb = 1;
    double beta = 0.0;
    double* C = nullptr;
    int64_t ldc = 1;
    int num_moduli = 16;
};

struct GemmConfig {
    int bn = 256, group_j = 16, ctas = 0;
};

// how gemm_adaptive picks s per tile (oz2_dgemm_adaptive modes)
enum class Adaptive { Mlp = 0, AnalyticTile = 1, AnalyticProblem = 2, Fixed = 3, CertifiedTile = 4, CertifiedProblem = 5 };
// the probe of Adaptive::Mlp (oz2_set_probe_kind)
enum class Probe { Columns = 0, Freivalds = 1, Both = 2, None = 3 };

struct AdaptiveStats {
    int64_t tiles = 0, sum_s = 0, probed = 0, rerun = 0, rerun_sum_s = 0, analytic_sum_s = 0, mlp = 0,
            int8_macs = 0, native_tiles = 0, native_macs = 0;
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
inline std::vector<oz2_dgemm_problem> problems(const std::vector<Problem>& ps) {
    std::vector<oz2_dgemm_problem> out(ps.size());
    for (size_t i = 0; i < ps.size(); ++i) {
        const Problem& p = ps[i];
        out[i] = oz2_dgemm_problem{op(p.ta), op(p.tb), p.num_moduli, p.m,   p.n, p.k,   p.alpha,
                                   p.beta,   p.A,      p.lda,        p.B,   p.ldb, p.C, p.ldc};
    }
    return out;
}
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

    // ---- beyond the reference: many problems in one set of launches, and adaptive s per tile

    // every problem as gemm() would compute it, bit for bit, in one grouped launch (problems with
    // num_moduli = OZ2_S_ADAPTIVE as gemm_adaptive(Mlp) would)
    void gemm_grouped(const std::vector<Problem>& ps, const std::vector<cudaEvent_t>& deps = {},
                      cudaEvent_t done = nullptr) {
        auto q = detail::problems(ps);
        std::vector<void*> d(deps.begin(), deps.end());
        detail::check(oz2_dgemm_grouped(h_, static_cast<int>(q.size()), q.data(), d.data(),
                                        static_cast<int>(d.size()), done),
                      h_);
    }
    void set_graph_mode(bool on) { detail::check(oz2_set_graph_mode(h_, on ? 1 : 0), h_); }
    void set_gemm_config(const GemmConfig& c) { detail::check(oz2_set_gemm_config(h_, c.bn, c.group_j, c.ctas), h_); }
    void clear_gemm_config() { detail::check(oz2_set_gemm_config(h_, 0, 0, 0), h_); }
    GemmConfig autotune_grouped(const std::vector<Problem>& ps) {
        auto q = detail::problems(ps);
        int v[3] = {0, 0, 0};
        detail::check(oz2_autotune_grouped(h_, static_cast<int>(q.size()), q.data(), v), h_);
        return GemmConfig{v[0], v[1], v[2]};
    }

    // C = alpha op(A) op(B) + beta C with s chosen per tile for `target_bits` (53: DGEMM-level
    // error); synchronises the stream
    AdaptiveStats gemm_adaptive(const std::vector<Problem>& ps, int target_bits = 53,
                                Adaptive mode = Adaptive::Mlp) {
        auto q = detail::problems(ps);
        int64_t v[10] = {};
        detail::check(oz2_dgemm_adaptive(h_, static_cast<int>(q.size()), q.data(), target_bits,
                                         static_cast<int>(mode), v),
                      h_);
        return AdaptiveStats{v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], v[8], v[9]};
    }
    // MLP parameters (the "params" array of a model file written by oz2.adaptive); empty unloads
    void set_mlp_weights(const std::vector<float>& params) {
        detail::check(oz2_mlp_set_weights(h_, params.empty() ? nullptr : params.data(), static_cast<int>(params.size())),
                      h_);
    }
    void set_adaptive_options(int tile, float threshold) {
        detail::check(oz2_set_adaptive_options(h_, tile, threshold), h_);
    }
    void set_probe_kind(Probe kind) { detail::check(oz2_set_probe_kind(h_, static_cast<int>(kind)), h_); }
    // {plane bytes read, residue bytes written, GEMM launches} of the last gemm_adaptive
    std::array<int64_t, 3> adaptive_gemm_bytes() const {
        std::array<int64_t, 3> v{};
        detail::check(oz2_adaptive_gemm_bytes(h_, v.data()), h_);
        return v;
    }

    // synchronises the stream; throws std::runtime_error if a kernel's bounded wait ran out
    void check_device_error() { detail::check(oz2_check_device_error(h_), h_); }

    oz2_handle handle() const { return h_; }

private:
    oz2_handle h_ = nullptr;
    Tuning tune_{};
};

}  // namespace oz2

namespace oz1 {

// The reference's Ozaki Scheme I comparison baseline (benchmarks/ozaki1_gpu.hpp:78-155) on this
// library's kernels: C = A B, column-major, untransposed, L 7-bit digits per element.
class Ozaki1 {
public:
    explicit Ozaki1(cudaStream_t stream = nullptr) { oz2::detail::check(oz2_create(stream, &h_)); }
    ~Ozaki1() { oz2_destroy(h_); }
    Ozaki1(const Ozaki1&) = delete;
    Ozaki1& operator=(const Ozaki1&) = delete;

    static int precision_bits(int L) { return 7 * L - 2; }
    static int num_gemms(int L) { return L * (L + 1) / 2; }

    // asynchronous on the stream; throws std::invalid_argument for L outside [2, 9] or k 4096 >= 2^31
    void gemm(int64_t m, int64_t n, int64_t k, const double* A, int64_t lda, const double* B, int64_t ldb, double* C,
              int64_t ldc, int L) {
        oz2::detail::check(oz2_ozaki1_dgemm(h_, m, n, k, A, lda, B, ldb, C, ldc, L), h_);
    }
    void release() { oz2::detail::check(oz2_release_workspace(h_), h_); }

private:
    oz2_handle h_ = nullptr;
};

}  // namespace oz1
