// ref_driver.cpp - C ABI over MacraMacra/OS2-Xe's own header src/ozaki2_gpu.hpp, compiled for the
// host against the CPU SYCL/oneMKL stand-in in oracle/ref_shim. The result, oracle/_ref/libozref.so,
// is the reference itself run here: the tests use it to pin the C oracle and to make golden
// vectors; bench.py --impl reference times it. TEST INFRASTRUCTURE ONLY.
#include <cstring>
#include <stdexcept>

#include "ozaki2_gpu.hpp"
#include "ozaki1_gpu.hpp"

namespace {
sycl::queue& q() {
    static sycl::queue qq(sycl::gpu_selector_v, sycl::property::queue::in_order());
    return qq;
}
oz2::Trans tr(char c) { return c == 'N' || c == 'n' ? oz2::Trans::N : (c == 'T' || c == 't' ? oz2::Trans::T : oz2::Trans::C); }

template <class F>
int guard(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::invalid_argument&) {
        return 1;
    } catch (const std::overflow_error&) {
        return 5;
    } catch (const std::exception&) {
        return 3;
    }
}
}  // namespace

extern "C" {

// plan (src/ozaki2_gpu.hpp:159-200): W is s x 8 words, M is 8 words
int ozref_make_plan(int s, int64_t k, int* tk, int* nl, double* log2M, uint32_t* m, uint32_t* y, uint32_t* W,
                    uint32_t* M) {
    return guard([&] {
        const oz2::detail::Plan p = oz2::detail::make_plan(s, k);
        *tk = p.tk;
        *nl = p.NL;
        *log2M = p.log2M;
        for (int t = 0; t < s; ++t) {
            m[t] = p.m[t];
            y[t] = p.y[t];
            std::memcpy(W + 8 * t, p.W[t].w, 8 * sizeof(uint32_t));
        }
        std::memcpy(M, p.M.w, 8 * sizeof(uint32_t));
    });
}

int ozref_precision_bits(int64_t k, int s, int* out) {
    return guard([&] { *out = oz2::Ozaki2::precision_bits(k, s); });
}
int ozref_moduli_for_bits(int64_t k, int bits) { return oz2::Ozaki2::moduli_for_bits(k, bits); }

// launch_split (src/ozaki2_gpu.hpp:407-455) on a column-major rows x cols matrix with ldx = rows;
// planes P[t*rows*cols + r + c*rows]; rows must be a multiple of 4. per_row selects ex[r] vs ex[c].
int ozref_split(int s, int tk, const double* X, int64_t rows, int64_t cols, const int* ex, int per_row, int8_t* P) {
    return guard([&] {
        using namespace oz2::detail;
        const Plan p = make_plan(s, 16);
        with_moduli(s, [&](auto S_) {
            constexpr int S = decltype(S_)::value;
            const SplitTab<S> tab = make_split_tab<S>(p);
            const bool wide = tk > oz2::kNarrowScaleBits;
            if (per_row) {
                if (wide) launch_split<S, true, 5>(q(), X, rows, rows, cols, ex, P, rows, rows * cols, tab, {}).wait();
                else launch_split<S, true, 3>(q(), X, rows, rows, cols, ex, P, rows, rows * cols, tab, {}).wait();
            } else {
                if (wide) launch_split<S, false, 5>(q(), X, rows, rows, cols, ex, P, rows, rows * cols, tab, {}).wait();
                else launch_split<S, false, 3>(q(), X, rows, rows, cols, ex, P, rows, rows * cols, tab, {}).wait();
            }
            return 0;
        });
    });
}

// launch_crt (src/ozaki2_gpu.hpp:603-626) for mb x nb outputs from Ct[t*mb*nb + i + j*mb]
int ozref_crt(int s, const int32_t* Ct, int64_t mb, int64_t nb, const int* D, const int* E, double alpha,
              double beta, double* C, int64_t ldc) {
    return guard([&] {
        using namespace oz2::detail;
        const Plan p = make_plan(s, 16);
        with_moduli(s, [&](auto S_) {
            constexpr int S = decltype(S_)::value;
            const CrtTab<S> tab = make_crt_tab<S>(p);
            launch_crt<S, false>(q(), Ct, mb * nb, 1, tab, mb, nb, D, E, alpha, beta, C, ldc, {}).wait();
            return 0;
        });
    });
}

// the full reference path, Ozaki2::gemm / zgemm (src/ozaki2_gpu.hpp:739-786)
int ozref_dgemm(char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A, int64_t lda,
                const double* B, int64_t ldb, double beta, double* C, int64_t ldc, int s, size_t ws_limit,
                int64_t* tiling) {
    return guard([&] {
        oz2::Ozaki2 oz(q());
        oz.set_workspace_limit(ws_limit);
        oz.gemm(tr(ta), tr(tb), m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s).wait();
        if (tiling) {
            const auto& t = oz.last_tiling();
            tiling[0] = t.mb; tiling[1] = t.nb; tiling[2] = t.pm; tiling[3] = t.pn; tiling[4] = t.k_chunks;
            tiling[5] = static_cast<int64_t>(t.workspace_bytes);
        }
    });
}

int ozref_zgemm(char ta, char tb, int64_t m, int64_t n, int64_t k, const double* alpha, const double* A,
                int64_t lda, const double* B, int64_t ldb, const double* beta, double* C, int64_t ldc, int s,
                size_t ws_limit) {
    return guard([&] {
        oz2::Ozaki2 oz(q());
        oz.set_workspace_limit(ws_limit);
        using cd = std::complex<double>;
        oz.zgemm(tr(ta), tr(tb), m, n, k, cd(alpha[0], alpha[1]), reinterpret_cast<const cd*>(A), lda,
                 reinterpret_cast<const cd*>(B), ldb, cd(beta[0], beta[1]), reinterpret_cast<cd*>(C), ldc, s)
            .wait();
    });
}

// the reference's Ozaki-I comparison baseline, oz1::Ozaki1::gemm (benchmarks/ozaki1_gpu.hpp:85-97)
int ozref_ozaki1(int64_t m, int64_t n, int64_t k, const double* A, int64_t lda, const double* B, int64_t ldb,
                 double* C, int64_t ldc, int L) {
    return guard([&] {
        oz1::Ozaki1 oz(q());
        oz.gemm(m, n, k, A, lda, B, ldb, C, ldc, L).wait();
    });
}

void ozref_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : 1);
#else
    (void)n;
#endif
}
}
