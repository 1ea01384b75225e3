// oz2_api.cu - the C ABI of liboz2.so (include/oz2/oz2.h) and the host orchestration of one
// emulated GEMM: argument checks, plan cache, tiling and workspace, then the phases
// scale -> split -> INT8 GEMM (+mod m) -> CRT on the handle's stream.
// Mirrors the reference's class oz2::Ozaki2 (src/ozaki2_gpu.hpp:678-1188); the internals are
// new: pre-tiled planes, tcgen05 products with residues fused, 1-byte residue planes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <utility>
#include <vector>

#include "../../include/oz2/oz2.h"
#include "oz2_kernels.cuh"
#include "oz2_plan.hpp"

using namespace oz2;

namespace {
enum Stage { kBegin = 0, kScale = 1, kSplit = 2, kGemm = 3, kCrt = 4 };
thread_local std::string g_error;  // errors of calls without a usable handle
}  // namespace

struct oz2_context {
    cudaStream_t stream = nullptr;
    int device = 0;
    int num_sms = 148;
    size_t ws_limit = 0, resident_hint = 0;
    uint8_t* ws = nullptr;
    size_t ws_size = 0;
    int* d_err = nullptr;
    Plan plan;
    int64_t plan_k = -1;
    int64_t tiling[6] = {0, 0, 0, 0, 0, 0};
    int tuning[3] = {1, 1, 1};
    bool profiling = false;
    std::vector<std::pair<int, cudaEvent_t>> marks;
    std::vector<cudaEvent_t> pool;
    size_t pool_used = 0;
    std::string err;
};

namespace {

int fail(oz2_context* h, int status, const std::string& msg) {
    if (h) h->err = msg;
    g_error = msg;
    return status;
}
int cuda_fail(oz2_context* h, cudaError_t e, const char* where) {
    return fail(h, OZ2_ECUDA, std::string("oz2: ") + where + ": " + cudaGetErrorString(e));
}
#define OZ2_CUDA(h, call)                                     \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, #call); \
    } while (0)

bool op_ok(char t) { return t == 'N' || t == 'n' || t == 'T' || t == 't' || t == 'C' || t == 'c'; }
bool is_n(char t) { return t == 'N' || t == 'n'; }
bool is_c(char t) { return t == 'C' || t == 'c'; }

void mark(oz2_context* h, int stage) {
    if (!h->profiling) return;
    if (h->pool_used == h->pool.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return;
        h->pool.push_back(e);
    }
    cudaEvent_t e = h->pool[h->pool_used++];
    cudaEventRecord(e, h->stream);
    h->marks.emplace_back(stage, e);
}

// ref src/ozaki2_gpu.hpp:745-748: dimensions and leading dimensions
int check_args(oz2_context* h, char ta, char tb, int64_t m, int64_t n, int64_t k, int64_t lda, int64_t ldb,
               int64_t ldc) {
    if (!op_ok(ta) || !op_ok(tb)) return fail(h, OZ2_EINVAL, "oz2: op must be 'N', 'T' or 'C'");
    if (m < 0 || n < 0 || k < 0) return fail(h, OZ2_EINVAL, "oz2: negative dimension");
    if (lda < std::max<int64_t>(1, is_n(ta) ? m : k) || ldb < std::max<int64_t>(1, is_n(tb) ? k : n) ||
        ldc < std::max<int64_t>(1, m))
        return fail(h, OZ2_EINVAL, "oz2: bad leading dimension");
    return OZ2_OK;
}

int begin_call(oz2_context* h, void* const* deps, int ndeps) {
    h->marks.clear();
    h->pool_used = 0;
    for (int i = 0; i < ndeps; ++i)
        if (deps && deps[i]) OZ2_CUDA(h, cudaStreamWaitEvent(h->stream, static_cast<cudaEvent_t>(deps[i]), 0));
    return OZ2_OK;
}
int end_call(oz2_context* h, void* done) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(h, e, "kernel launch");
    if (done) OZ2_CUDA(h, cudaEventRecord(static_cast<cudaEvent_t>(done), h->stream));
    return OZ2_OK;
}

int ensure_plan(oz2_context* h, int s, int64_t k) {
    if (h->plan.s == s && h->plan_k == k) return OZ2_OK;
    Plan p;
    const int st = make_plan(s, k, p);
    if (st) {
        char buf[160];
        plan_error_text(s, k, st, buf, sizeof buf);
        return fail(h, st == 5 ? OZ2_EOVERFLOW : (st == 1 ? OZ2_EINVAL : OZ2_EINTERNAL), buf);
    }
    h->plan = p;
    h->plan_k = k;
    return OZ2_OK;
}

// ---------------------------------------------------------------- tiling / workspace
struct Layout {
    int64_t mb, nb, pm, pn, kchunks;
    size_t bytes;
    size_t o_maxA, o_maxB, o_A, o_B, o_R;
};

size_t align256(size_t v) { return (v + 255) & ~size_t{255}; }

Layout layout_for(int64_t m, int64_t n, int64_t k, int s, int G, int64_t mb, int64_t nb) {
    Layout L{};
    L.mb = mb;
    L.nb = nb;
    L.pm = ceil_div(m, mb);
    L.pn = ceil_div(n, nb);
    const int64_t kb = ceil_div(k, kTileK);
    L.kchunks = ceil_div(kb, kChunkKB);
    const PlaneGeom ga = plane_geom(mb, k, kGemmI), gb = plane_geom(nb, k, kGemmJ);
    const int64_t ldr = round_up(mb, 32);
    size_t off = 0;
    auto carve = [&](size_t bytes) {
        const size_t o = off;
        off = align256(off + bytes);
        return o;
    };
    L.o_maxA = carve(static_cast<size_t>(m) * 8);
    L.o_maxB = carve(static_cast<size_t>(n) * 8);
    L.o_A = carve(static_cast<size_t>(G) * s * ga.plane_bytes);
    L.o_B = carve(static_cast<size_t>(G) * s * gb.plane_bytes);
    L.o_R = carve(static_cast<size_t>(G) * s * nb * ldr);
    L.bytes = off;
    return L;
}

size_t budget(oz2_context* h) {
    if (h->ws_limit) return h->ws_limit;
    size_t free_b = 0, total = 0;
    if (cudaMemGetInfo(&free_b, &total) != cudaSuccess) return 0;
    free_b += h->ws_size;  // the current workspace is reusable
    const size_t reserve = (size_t{512} << 20) + total / 32;
    size_t lim = free_b > reserve ? free_b - reserve : 0;
    if (h->resident_hint)
        lim = std::min(lim, total > reserve + h->resident_hint ? total - reserve - h->resident_hint : size_t{0});
    return lim;
}

std::vector<int64_t> tile_candidates(int64_t x, int64_t unit, bool pow2) {
    std::vector<int64_t> c{x};
    for (int64_t p = 2; p <= 256; ++p) {
        const int64_t b = round_up(ceil_div(x, p), unit);
        if (b < x) c.push_back(b);
    }
    if (pow2)
        for (int64_t b = 1024; b < x; b *= 2) c.push_back(b);
    std::sort(c.begin(), c.end(), std::greater<>());
    c.erase(std::unique(c.begin(), c.end()), c.end());
    return c;
}

// Largest column tile that fits for each row-tile candidate, scored by an analytic time model
// of this implementation (tensor-core work on padded tiles, HBM traffic of split and CRT,
// per-launch overhead).
int choose_layout(oz2_context* h, int64_t m, int64_t n, int64_t k, int s, int G, Layout& out) {
    const size_t limit = budget(h);
    double best = std::numeric_limits<double>::infinity();
    const bool pow2 = h->tuning[2] != 0;
    const auto nbs = tile_candidates(n, kGemmJ, pow2);
    for (int64_t mb : tile_candidates(m, kGemmI, pow2)) {
        for (int64_t nb : nbs) {
            const Layout L = layout_for(m, n, k, s, G, mb, nb);
            if (L.bytes > limit) continue;
            const double gemm = 2.0 * G * s * k * static_cast<double>(L.pm * round_up(mb, kGemmI)) *
                                static_cast<double>(L.pn * round_up(nb, kGemmJ)) / 3.0e15;
            const double split = G * (8.0 + s) * (static_cast<double>(k) * m * (L.pm > 1 ? L.pn : 1) +
                                                  static_cast<double>(k) * n) / 5.0e12;
            const double crt = G * (s + 16.0) * static_cast<double>(m) * n / 5.0e12;
            const double t = gemm + split + crt + L.pm * L.pn * (L.kchunks + 3) * 5e-6;
            if (t < best) {
                best = t;
                out = L;
            }
            break;
        }
    }
    if (!std::isfinite(best)) {
        char buf[128];
        std::snprintf(buf, sizeof buf, "oz2: not enough device memory for workspace (limit %zu MiB)", limit >> 20);
        return fail(h, OZ2_ENOMEM, buf);
    }
    return OZ2_OK;
}

int ensure_workspace(oz2_context* h, size_t bytes) {
    if (h->ws_size >= bytes) return OZ2_OK;
    OZ2_CUDA(h, cudaStreamSynchronize(h->stream));
    if (h->ws) cudaFree(h->ws);
    h->ws = nullptr;
    h->ws_size = 0;
    if (cudaMalloc(&h->ws, bytes) != cudaSuccess) {
        cudaGetLastError();
        h->ws = nullptr;
        return fail(h, OZ2_ENOMEM, "oz2: workspace allocation failed");
    }
    h->ws_size = bytes;
    return OZ2_OK;
}

// ---------------------------------------------------------------- one emulated GEMM
// G = 1: real; G = 3: complex 3M (groups re, im, re+im). X pointers are double* views.
int run(oz2_context* h, char ta, char tb, int64_t m, int64_t n, int64_t k, const double* alpha, const double* A,
        int64_t lda, const double* B, int64_t ldb, const double* beta, double* C, int64_t ldc, int G) {
    const Plan& p = h->plan;
    const int s = p.s;
    const bool cplx = G == 3;
    ModConst mc[kMaxModuli];
    mod_constants(p, mc);
    Layout L;
    int st = choose_layout(h, m, n, k, s, G, L);
    if (st) return st;
    if ((st = ensure_workspace(h, L.bytes))) return st;
    h->tiling[0] = L.mb;
    h->tiling[1] = L.nb;
    h->tiling[2] = L.pm;
    h->tiling[3] = L.pn;
    h->tiling[4] = L.kchunks;
    h->tiling[5] = static_cast<int64_t>(L.bytes);

    auto* maxA = reinterpret_cast<unsigned long long*>(h->ws + L.o_maxA);
    auto* maxB = reinterpret_cast<unsigned long long*>(h->ws + L.o_maxB);
    auto* planesA = reinterpret_cast<int8_t*>(h->ws + L.o_A);
    auto* planesB = reinterpret_cast<int8_t*>(h->ws + L.o_B);
    auto* resid = h->ws + L.o_R;
    const int w = cplx ? 2 : 1;
    const int64_t kb_total = ceil_div(k, kTileK);
    const int64_t ldr = round_up(L.mb, 32);
    if (kb_total > 65535 * 4 || (kb_total > 65535 && (is_n(ta) || !is_n(tb))))
        return fail(h, OZ2_EINVAL, "oz2: k too large for one call of this implementation");

    mark(h, kBegin);
    OZ2_CUDA(h, cudaMemsetAsync(maxA, 0, static_cast<size_t>(m) * 8, h->stream));
    OZ2_CUDA(h, cudaMemsetAsync(maxB, 0, static_cast<size_t>(n) * 8, h->stream));
    // A side: plane rows are rows i of op(A); B side: plane rows are columns j of op(B)
    SideDesc sa{A, lda, m, k, is_n(ta), cplx, cplx && is_c(ta)};
    SideDesc sb{B, ldb, n, k, !is_n(tb), cplx, cplx && is_c(tb)};
    launch_scale(sa, maxA, h->num_sms, h->stream);
    launch_scale(sb, maxB, h->num_sms, h->stream);
    mark(h, kScale);

    for (int64_t j0 = 0; j0 < n; j0 += L.nb) {
        const int64_t nbj = std::min(L.nb, n - j0);
        const PlaneGeom gb = plane_geom(nbj, k, kGemmJ);
        SideDesc tb_side = sb;
        tb_side.X = B + w * (sb.row_contig ? j0 : j0 * ldb);
        tb_side.rows = nbj;
        launch_split(tb_side, maxB + j0, p.tk, mc, s, planesB, gb, h->stream);
        mark(h, kSplit);
        for (int64_t i0 = 0; i0 < m; i0 += L.mb) {
            const int64_t mbi = std::min(L.mb, m - i0);
            const PlaneGeom ga = plane_geom(mbi, k, kGemmI);
            if (L.pm > 1 || j0 == 0) {
                SideDesc ta_side = sa;
                ta_side.X = A + w * (sa.row_contig ? i0 : i0 * lda);
                ta_side.rows = mbi;
                launch_split(ta_side, maxA + i0, p.tk, mc, s, planesA, ga, h->stream);
                mark(h, kSplit);
            }
            for (int64_t c = 0; c < L.kchunks; ++c) {
                GemmArgs g{};
                g.planes_i = planesA;
                g.planes_j = planesB;
                g.resid = resid;
                g.pstride_i = ga.plane_bytes;
                g.pstride_j = gb.plane_bytes;
                g.rstride = L.nb * ldr;
                g.ldr = ldr;
                g.m = mbi;
                g.n = nbj;
                g.kb_total = kb_total;
                g.kb0 = c * kChunkKB;
                g.kb1 = std::min(kb_total, g.kb0 + kChunkKB);
                g.s = s;
                g.groups = G;
                g.accumulate = c > 0;
                g.mc = mc;
                g.err = h->d_err;
                launch_gemm(g, h->num_sms, h->stream);
            }
            mark(h, kGemm);
            CrtArgs ca{};
            ca.resid = resid;
            ca.rstride = L.nb * ldr;
            ca.ldr = ldr;
            ca.m = mbi;
            ca.n = nbj;
            ca.maxA = maxA + i0;
            ca.maxB = maxB + j0;
            ca.tk = p.tk;
            ca.cplx = cplx;
            ca.alpha[0] = alpha[0];
            ca.alpha[1] = cplx ? alpha[1] : 0.0;
            ca.beta[0] = beta[0];
            ca.beta[1] = cplx ? beta[1] : 0.0;
            ca.C = C + w * (i0 + j0 * ldc);
            ca.ldc = ldc;
            ca.plan = &p;
            launch_crt(ca, h->stream);
            mark(h, kCrt);
        }
    }
    return OZ2_OK;
}

}  // namespace

namespace oz2 {
// lets entry points without a handle report a message through oz2_last_error(NULL)
void set_last_error(const std::string& msg) { g_error = msg; }
}  // namespace oz2

extern "C" {

int oz2_create(void* stream, oz2_handle* out) {
    if (!out) return fail(nullptr, OZ2_EINVAL, "oz2: null output handle");
    auto* h = new oz2_context;
    h->stream = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaGetDevice(&h->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(h->d_err, 0, sizeof(int));
    if (e != cudaSuccess) {
        const int st = cuda_fail(nullptr, e, "oz2_create");
        if (h->d_err) cudaFree(h->d_err);
        delete h;
        *out = nullptr;
        return st;
    }
    *out = h;
    return OZ2_OK;
}

int oz2_destroy(oz2_handle h) {
    if (!h) return OZ2_OK;
    cudaStreamSynchronize(h->stream);
    if (h->ws) cudaFree(h->ws);
    if (h->d_err) cudaFree(h->d_err);
    for (cudaEvent_t e : h->pool) cudaEventDestroy(e);
    delete h;
    return OZ2_OK;
}

int oz2_set_stream(oz2_handle h, void* stream) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    h->stream = static_cast<cudaStream_t>(stream);
    return OZ2_OK;
}

// ref src/ozaki2_gpu.hpp:739-760
int oz2_dgemm(oz2_handle h, char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A,
              int64_t lda, const double* B, int64_t ldb, double beta, double* C, int64_t ldc, int num_moduli,
              void* const* deps, int ndeps, void* done) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    h->marks.clear();
    int st = check_args(h, ta, tb, m, n, k, lda, ldb, ldc);
    if (st) return st;
    if ((st = begin_call(h, deps, ndeps))) return st;
    if (m == 0 || n == 0) return end_call(h, done);
    const double al[2] = {alpha, 0.0}, be[2] = {beta, 0.0};
    if (k == 0 || alpha == 0.0) {
        launch_scale_c(C, ldc, m, n, be, false, h->stream);
        return end_call(h, done);
    }
    if ((st = ensure_plan(h, num_moduli, k))) return st;
    if ((st = run(h, ta, tb, m, n, k, al, A, lda, B, ldb, be, C, ldc, 1))) return st;
    return end_call(h, done);
}

// ref src/ozaki2_gpu.hpp:764-786 (plan for 2k: the 3M sums double the inner products)
int oz2_zgemm(oz2_handle h, char ta, char tb, int64_t m, int64_t n, int64_t k, const double* alpha,
              const double* A, int64_t lda, const double* B, int64_t ldb, const double* beta, double* C,
              int64_t ldc, int num_moduli, void* const* deps, int ndeps, void* done) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    if (!alpha || !beta) return fail(h, OZ2_EINVAL, "oz2: null alpha or beta");
    h->marks.clear();
    int st = check_args(h, ta, tb, m, n, k, lda, ldb, ldc);
    if (st) return st;
    if ((st = begin_call(h, deps, ndeps))) return st;
    if (m == 0 || n == 0) return end_call(h, done);
    if (k == 0 || (alpha[0] == 0.0 && alpha[1] == 0.0)) {
        launch_scale_c(C, ldc, m, n, beta, true, h->stream);
        return end_call(h, done);
    }
    if (k > std::numeric_limits<int64_t>::max() / 2) return fail(h, OZ2_EINVAL, "oz2: k too large");
    if ((st = ensure_plan(h, num_moduli, 2 * k))) return st;
    if ((st = run(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, 3))) return st;
    return end_call(h, done);
}

int oz2_precision_bits(int64_t k, int num_moduli, int* out) {
    Plan p;
    const int st = make_plan(num_moduli, k, p);
    if (st) {
        char buf[160];
        return fail(nullptr, st == 1 ? OZ2_EINVAL : OZ2_EINTERNAL, plan_error_text(num_moduli, k, st, buf, sizeof buf));
    }
    if (out) *out = p.tk;
    return OZ2_OK;
}

int oz2_precision_bits_complex(int64_t k, int num_moduli, int* out) {
    if (k > std::numeric_limits<int64_t>::max() / 2) return fail(nullptr, OZ2_EINVAL, "oz2: k too large");
    return oz2_precision_bits(2 * k, num_moduli, out);
}

// ref src/ozaki2_gpu.hpp:693-700: smallest s whose tk reaches `bits`, else 24
int oz2_moduli_for_bits(int64_t k, int bits, int* out) {
    int best = kMaxModuli;
    for (int s = 2; s <= kMaxModuli; ++s) {
        Plan p;
        if (make_plan(s, k, p) == 0 && p.tk >= bits) {
            best = s;
            break;
        }
    }
    if (out) *out = best;
    return OZ2_OK;
}

int oz2_set_workspace_limit(oz2_handle h, size_t bytes) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    h->ws_limit = bytes;
    return OZ2_OK;
}
int oz2_set_resident_hint(oz2_handle h, size_t bytes) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    h->resident_hint = bytes;
    return OZ2_OK;
}
int oz2_release_workspace(oz2_handle h) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    if (!h->ws) return OZ2_OK;
    OZ2_CUDA(h, cudaStreamSynchronize(h->stream));
    cudaFree(h->ws);
    h->ws = nullptr;
    h->ws_size = 0;
    return OZ2_OK;
}

int oz2_set_profiling(oz2_handle h, int enable) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    h->profiling = enable != 0;
    return OZ2_OK;
}

// ref src/ozaki2_gpu.hpp:716-737: each stage gets the time from the previous mark to its own
int oz2_stage_times(oz2_handle h, double* out4) {
    if (!h || !out4) return fail(h, OZ2_EINVAL, "oz2: null argument");
    for (int i = 0; i < 4; ++i) out4[i] = 0.0;
    if (!h->profiling || h->marks.empty()) return OZ2_OK;
    OZ2_CUDA(h, cudaEventSynchronize(h->marks.back().second));
    for (size_t i = 1; i < h->marks.size(); ++i) {
        float ms = 0.0f;
        OZ2_CUDA(h, cudaEventElapsedTime(&ms, h->marks[i - 1].second, h->marks[i].second));
        const int stg = h->marks[i].first;
        if (stg >= kScale && stg <= kCrt) out4[stg - 1] += ms;
    }
    return OZ2_OK;
}

int oz2_last_tiling(oz2_handle h, int64_t* out6) {
    if (!h || !out6) return fail(h, OZ2_EINVAL, "oz2: null argument");
    for (int i = 0; i < 6; ++i) out6[i] = h->tiling[i];
    return OZ2_OK;
}

int oz2_set_tuning(oz2_handle h, int batched_gemm, int pad_lda, int pow2_tiles) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    h->tuning[0] = batched_gemm;
    h->tuning[1] = pad_lda;
    h->tuning[2] = pow2_tiles;
    return OZ2_OK;
}

int oz2_check_device_error(oz2_handle h) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    OZ2_CUDA(h, cudaStreamSynchronize(h->stream));
    int v = 0;
    OZ2_CUDA(h, cudaMemcpy(&v, h->d_err, sizeof v, cudaMemcpyDeviceToHost));
    if (v) {
        OZ2_CUDA(h, cudaMemset(h->d_err, 0, sizeof v));
        char buf[96];
        std::snprintf(buf, sizeof buf, "oz2: a device-side wait ran out (code %d)", v);
        return fail(h, OZ2_ETIMEOUT, buf);
    }
    return OZ2_OK;
}

const char* oz2_last_error(oz2_handle h) { return h ? h->err.c_str() : g_error.c_str(); }

const char* oz2_status_string(int status) {
    switch (status) {
        case OZ2_OK: return "ok";
        case OZ2_EINVAL: return "invalid argument";
        case OZ2_ENOMEM: return "out of device memory";
        case OZ2_EINTERNAL: return "internal error";
        case OZ2_ETIMEOUT: return "device-side wait timed out";
        case OZ2_EOVERFLOW: return "overflow";
        case OZ2_ECUDA: return "CUDA error";
    }
    return "unknown status";
}

}  // extern "C"
