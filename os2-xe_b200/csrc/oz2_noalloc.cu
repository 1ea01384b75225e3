// oz2_noalloc.cu - oz2_dgemm_noalloc: the emulated DGEMM for callers that cannot allocate device
// memory. The reference has no counterpart.
//
// Who needs it: code that runs where cudaMalloc is unavailable or forbidden, e.g. inside a
// memory-pool owner that must not see foreign allocations, a real-time loop that may not call
// the driver's allocator, or a plugin host that hands out only the buffers of its inputs and
// outputs. oz2_dgemm keeps a workspace that it grows with cudaMalloc; this entry point instead
// carves its scratch (row/column maxima, INT8 planes, residues, device error word) out of one
// file-scope static __device__ array of kScratchBytes bytes, and allocates nothing itself: no
// cudaMalloc, no cudaFree, no allocating library routine. The caller passes inputs and outputs.
//
// Cost of that choice: every GPU that loads this part of the library holds the array until
// the process exits, and the problem must fit in it (checked; larger problems are rejected with
// OZ2_EINVAL). All calls share the one array, which keeps the last call's contents: each call
// clears the regions that must start at zero, and calls that overlap on the GPU (on different
// streams, or from different host threads without ordering) race on it.
//
// Set-up: the first call on each device looks up the device address of the array with
// cudaGetSymbolAddress while that device is current (in host code the array's name is only a
// host-side stand-in). That first call should come before any stream capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/oz2/oz2.h"
#include "oz2_kernels.cuh"
#include "oz2_plan.hpp"

namespace oz2 {
void set_last_error(const std::string& msg);  // defined in oz2_api.cu
}

namespace {

constexpr size_t kScratchBytes = size_t{64} << 20;  // the stated maximum: 64 MiB
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_dev[kMaxDevices] = {};
int g_num_sms[kMaxDevices] = {};

int reject(int status, const std::string& msg) {
    oz2::set_last_error(msg);
    return status;
}

// once per device, with that device current
int scratch_for_current_device(unsigned char** ptr, int* num_sms) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return reject(OZ2_ECUDA, std::string("oz2_dgemm_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return reject(OZ2_EINVAL, "oz2_dgemm_noalloc: device index out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_dev[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p)
            return reject(OZ2_ECUDA, std::string("oz2_dgemm_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return reject(OZ2_ECUDA, std::string("oz2_dgemm_noalloc: ") + cudaGetErrorString(e));
        g_num_sms[dev] = sms;
        g_scratch_dev[dev] = static_cast<unsigned char*>(p);
    }
    *ptr = g_scratch_dev[dev];
    *num_sms = g_num_sms[dev];
    return OZ2_OK;
}

bool is_n(char t) { return t == 'N' || t == 'n'; }
bool op_ok(char t) { return t == 'N' || t == 'n' || t == 'T' || t == 't' || t == 'C' || t == 'c'; }
size_t align256(size_t v) { return (v + 255) & ~size_t{255}; }

}  // namespace

extern "C" int oz2_dgemm_noalloc(void* stream, char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha,
                                 const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
                                 int64_t ldc, int num_moduli) {
    using namespace oz2;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the same checks, in the same order, as oz2_dgemm
    if (!op_ok(ta) || !op_ok(tb)) return reject(OZ2_EINVAL, "oz2: op must be 'N', 'T' or 'C'");
    if (m < 0 || n < 0 || k < 0) return reject(OZ2_EINVAL, "oz2: negative dimension");
    if (lda < std::max<int64_t>(1, is_n(ta) ? m : k) || ldb < std::max<int64_t>(1, is_n(tb) ? k : n) ||
        ldc < std::max<int64_t>(1, m))
        return reject(OZ2_EINVAL, "oz2: bad leading dimension");
    if (m == 0 || n == 0) return OZ2_OK;
    if (k == 0 || alpha == 0.0) {
        const double be[2] = {beta, 0.0};
        launch_scale_c(C, ldc, m, n, be, false, st);
        const cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? OZ2_OK : reject(OZ2_ECUDA, std::string("oz2: ") + cudaGetErrorString(e));
    }
    Plan p;
    const int ps = make_plan(num_moduli, k, p);
    if (ps) {
        char buf[160];
        return reject(ps == 1 ? OZ2_EINVAL : OZ2_EINTERNAL, plan_error_text(num_moduli, k, ps, buf, sizeof buf));
    }
    const int s = p.s;
    const PlaneGeom ga = plane_geom(m, k, kGemmI), gb = plane_geom(n, k, kGemmJ);
    const int64_t ldr = round_up(m, 32);
    const int64_t kb_total = ga.kb_total;
    if (kb_total > 65535 * 4 || (kb_total > 65535 && (is_n(ta) || !is_n(tb))))
        return reject(OZ2_EINVAL, "oz2: k too large for one call of this implementation");
    // scratch layout: error word | maxA | maxB | planes A | planes B | residues
    const size_t o_err = 0;
    const size_t o_maxA = 256;
    const size_t o_maxB = align256(o_maxA + static_cast<size_t>(m) * 8);
    const size_t o_A = align256(o_maxB + static_cast<size_t>(n) * 8);
    const size_t o_B = align256(o_A + static_cast<size_t>(s) * ga.plane_bytes);
    const size_t o_R = align256(o_B + static_cast<size_t>(s) * gb.plane_bytes);
    const size_t need = align256(o_R + static_cast<size_t>(s) * n * ldr);
    if (need > kScratchBytes) {
        char buf[200];
        std::snprintf(buf, sizeof buf,
                      "oz2_dgemm_noalloc: this problem needs %zu bytes of scratch; the static scratch holds %zu "
                      "bytes (64 MiB): use oz2_dgemm",
                      need, kScratchBytes);
        return reject(OZ2_EINVAL, buf);
    }
    unsigned char* scratch = nullptr;
    int num_sms = 0;
    int rc = scratch_for_current_device(&scratch, &num_sms);
    if (rc) return rc;

    auto* err = reinterpret_cast<int*>(scratch + o_err);
    auto* maxA = reinterpret_cast<unsigned long long*>(scratch + o_maxA);
    auto* maxB = reinterpret_cast<unsigned long long*>(scratch + o_maxB);
    auto* planesA = reinterpret_cast<int8_t*>(scratch + o_A);
    auto* planesB = reinterpret_cast<int8_t*>(scratch + o_B);
    unsigned char* resid = scratch + o_R;
    // the array keeps the previous call's contents: the error word and the maxima must start at
    // zero; planes and residues are overwritten in full by the split and the first k chunk
    cudaError_t e = cudaMemsetAsync(scratch, 0, o_A, st);
    if (e != cudaSuccess) return reject(OZ2_ECUDA, std::string("oz2_dgemm_noalloc: ") + cudaGetErrorString(e));

    ModConst mc[kMaxModuli];
    mod_constants(p, mc);
    SideDesc sa{A, lda, m, k, is_n(ta), false, false};
    SideDesc sb{B, ldb, n, k, !is_n(tb), false, false};
    launch_scale(sa, maxA, num_sms, st);
    launch_scale(sb, maxB, num_sms, st);
    launch_split(sb, maxB, p.tk, mc, s, planesB, gb, st);
    launch_split(sa, maxA, p.tk, mc, s, planesA, ga, st);
    const int64_t chunks = ceil_div(kb_total, kChunkKB);
    for (int64_t c = 0; c < chunks; ++c) {
        GemmArgs g{};
        g.planes_i = planesA;
        g.planes_j = planesB;
        g.resid = resid;
        g.pstride_i = ga.plane_bytes;
        g.pstride_j = gb.plane_bytes;
        g.rstride = n * ldr;
        g.ldr = ldr;
        g.m = m;
        g.n = n;
        g.kb_total = kb_total;
        g.kb0 = c * kChunkKB;
        g.kb1 = std::min(kb_total, g.kb0 + kChunkKB);
        g.s = s;
        g.groups = 1;
        g.accumulate = c > 0;
        g.mc = mc;
        g.err = err;
        launch_gemm(g, num_sms, st);
    }
    CrtArgs ca{};
    ca.resid = resid;
    ca.rstride = n * ldr;
    ca.ldr = ldr;
    ca.m = m;
    ca.n = n;
    ca.maxA = maxA;
    ca.maxB = maxB;
    ca.tk = p.tk;
    ca.cplx = false;
    ca.alpha[0] = alpha;
    ca.beta[0] = beta;
    ca.C = C;
    ca.ldc = ldc;
    ca.plan = &p;
    launch_crt(ca, st);
    e = cudaGetLastError();
    return e == cudaSuccess ? OZ2_OK : reject(OZ2_ECUDA, std::string("oz2_dgemm_noalloc: ") + cudaGetErrorString(e));
}
