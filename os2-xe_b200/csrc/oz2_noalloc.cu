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
// host-side stand-in) and raises the GEMM kernels' dynamic shared-memory limit, which a process
// that never created a handle has not done. That first call should come before any stream
// capture. The address is kept per device for the life of the process: after cudaDeviceReset
// the array may move, so this entry point must not be used after a device reset.
//
// Errors on the device: the GEMM's bounded waits record a code in the first word of the array.
// oz2_noalloc_check_device_error reads (and clears) it; the next call clears it too, so check
// after the call whose result matters and before the next one.
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
        // the GEMM needs more than 48 KiB of dynamic shared memory; oz2_create sets this for
        // handle users, and a caller of this entry point may never have created a handle
        e = oz2::prepare_gemm_kernels();
        if (e != cudaSuccess)
            return reject(OZ2_ECUDA, std::string("oz2_dgemm_noalloc: kernel set-up: ") + cudaGetErrorString(e));
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
    const PlaneGeom ga = plane_geom(m, k, kGemmIPad), gb = plane_geom(n, k, kGemmJ);
    const int64_t ldr = round_up(m, 32);
    const int64_t kb_total = ga.kb_total;
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
    const size_t o_D = need;  // item tables after the buffers
    const size_t desc_need = o_D + 8 * 1024;
    if (desc_need > kScratchBytes) {
        char buf[200];
        std::snprintf(buf, sizeof buf,
                      "oz2_dgemm_noalloc: this problem needs %zu bytes of scratch; the static scratch holds %zu "
                      "bytes (64 MiB): use oz2_dgemm",
                      desc_need, kScratchBytes);
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

    // item tables (one problem), written into the scratch by a kernel that takes them as its
    // parameter: host memory only, no staging buffer
    ModConst mc[kMaxModuliExt];
    mod_constants(p, mc);
    struct Tables {
        ScaleItem sc[2];
        SplitItem sp[2];
        GemmItem g;
        CrtItem c;
    };
    static thread_local Tables T;
    T = Tables{};
    for (int side = 0; side < 2; ++side) {
        ScaleItem& si = T.sc[side];
        si.X = side ? B : A;
        si.ldx = side ? ldb : lda;
        si.rows = side ? n : m;
        si.k = k;
        si.row_contig = side ? !is_n(tb) : is_n(ta);
        si.out = side ? maxB : maxA;
        scale_item_blocks(si, num_sms, 0);
        SplitItem& sp = T.sp[side];
        sp.X = si.X;
        sp.ldx = si.ldx;
        sp.rows = si.rows;
        sp.k = k;
        sp.row_contig = si.row_contig;
        sp.tk = p.tk;
        sp.s = s;
        sp.maxbits = si.out;
        sp.planes = side ? planesB : planesA;
        const PlaneGeom& gg = side ? gb : ga;
        sp.plane_bytes = gg.plane_bytes;
        sp.kb_total = gg.kb_total;
        sp.rows_pad = gg.rows_pad;
        for (int t = 0; t < s; ++t) sp.mc[t] = mc[t];
        split_geometry(sp, 0);
    }
    GemmConfig cfg;
    cfg.bn = m <= 384 ? 128 : 256;
    GemmItem& g = T.g;
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
    g.tiles_i = static_cast<int>(gemm_tiles_i(m, cfg.bn));
    g.tiles_j = static_cast<int>(ceil_div(n, kGemmJ));
    g.tiles = static_cast<int64_t>(g.tiles_i) * g.tiles_j;
    g.s = s;
    g.groups = 1;
    g.job0 = 0;
    for (int t = 0; t < s; ++t) {
        g.mod_m[t] = mc[t].m;
        g.mod_mu[t] = mc[t].mu;
        g.mod_kbias[t] = mc[t].kbias;
        g.mod_kbias30[t] = mc[t].kbias30;
        g.mod_mx31[t] = mc[t].mx31;
        g.mod_mxs[t] = mc[t].mxs;
    }
    CrtItem& c = T.c;
    c.resid = resid;
    c.rstride = n * ldr;
    c.gstride = c.rstride * s;
    c.ldr = ldr;
    c.m = m;
    c.n = n;
    c.ldc = ldc;
    c.maxA = maxA;
    c.maxB = maxB;
    c.tk = p.tk;
    c.ar = alpha;
    c.br = beta;
    c.C = C;
    c.mma = crt_uses_mma(p, false) ? 1 : 0;
    const int64_t crt_blocks = crt_item_blocks(c, 0);
    static_assert(sizeof(Tables) <= 8 * 1024, "item tables exceed their scratch region");
    unsigned char* dtab = scratch + o_D;
    launch_write_blob(&T, sizeof(Tables), dtab, st);
    const Tables* D = reinterpret_cast<const Tables*>(dtab);
    for (int side = 0; side < 2; ++side)
        launch_scale(&D->sc[side], &T.sc[side], 1, T.sc[side].rblocks * ceil_div(k, T.sc[side].kchunk), st);
    for (int side = 1; side >= 0; --side)
        launch_split(&D->sp[side], &T.sp[side], 1, T.sp[side].rblocks * T.sp[side].kblocks, err, st);
    launch_gemm(&D->g, 1, g.tiles * s, cfg, num_sms, err, st);
    launch_crt(&D->c, 1, crt_blocks, p, false, err, st);
    e = cudaGetLastError();
    return e == cudaSuccess ? OZ2_OK : reject(OZ2_ECUDA, std::string("oz2_dgemm_noalloc: ") + cudaGetErrorString(e));
}

extern "C" int oz2_noalloc_check_device_error(void* stream) {
    using namespace oz2;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char* scratch = nullptr;
    int num_sms = 0;
    const int rc = scratch_for_current_device(&scratch, &num_sms);
    if (rc) return rc;
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return reject(OZ2_ECUDA, std::string("oz2_noalloc_check_device_error: ") + cudaGetErrorString(e));
    int v = 0;
    e = cudaMemcpy(&v, scratch, sizeof v, cudaMemcpyDeviceToHost);  // the error word at offset 0
    if (e != cudaSuccess) return reject(OZ2_ECUDA, std::string("oz2_noalloc_check_device_error: ") + cudaGetErrorString(e));
    if (v) {
        e = cudaMemset(scratch, 0, sizeof v);
        if (e != cudaSuccess)
            return reject(OZ2_ECUDA, std::string("oz2_noalloc_check_device_error: ") + cudaGetErrorString(e));
        char buf[96];
        std::snprintf(buf, sizeof buf, "oz2_dgemm_noalloc: a device-side wait ran out (code %d)", v);
        return reject(OZ2_ETIMEOUT, buf);
    }
    return OZ2_OK;
}
