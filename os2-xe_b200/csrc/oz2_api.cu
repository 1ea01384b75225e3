// oz2_api.cu - the C ABI of liboz2.so (include/oz2/oz2.h) and the host orchestration of the
// emulated GEMMs: argument checks, plan cache, tiling and workspace, descriptor tables, then
// the phases scale -> split -> INT8 GEMM (+mod m) -> CRT on the handle's stream.
// Mirrors the reference's class oz2::Ozaki2 (src/ozaki2_gpu.hpp:678-1188) for single calls and
// adds a grouped call (many independent DGEMMs in one set of launches, optionally replayed
// from a CUDA graph) with a GEMM-configuration autotuner; the reference has neither.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "../../include/oz2/oz2.h"
#include "oz2_adaptive.cuh"
#include "oz2_kernels.cuh"
#include "oz2_plan.hpp"

using namespace oz2;

namespace {
enum Stage { kBegin = 0, kScale = 1, kSplit = 2, kGemm = 3, kCrt = 4, kProbe = 5, kNative = 6 };
thread_local std::string g_error;  // errors of calls without a usable handle
constexpr int kRing = 4;

// ---------------------------------------------------------------- launch program of one call
// A call is planned on the host into a descriptor blob and a list of operations, then issued
// on the stream (or captured into a CUDA graph and replayed).
struct Op {
    enum Kind { Memset, Scale, Split, Gemm, Crt, ScaleC, Mark, Slice, GemmOz1, GemmCrt } kind;
    size_t off = 0;    // descriptor offset in the blob
    int count = 0;     // items
    int64_t blocks = 0;
    void* ptr = nullptr;
    size_t bytes = 0;  // memset
    const Plan* plan = nullptr;
    bool cplx = false;
    GemmConfig cfg;
    int64_t jobs = 0;
    int64_t m = 0, n = 0, ldc = 0;  // scale_c
    double beta[2] = {0, 0};
    int stage = 0;
};

struct Program {
    std::vector<unsigned char> blob;
    std::vector<Op> ops;
    size_t add(const void* p, size_t bytes) {
        const size_t off = (blob.size() + 255) & ~size_t{255};
        blob.resize(off + bytes);
        std::memcpy(blob.data() + off, p, bytes);
        return off;
    }
};

// one grouped call captured for replay: an executable graph per batch of problems, the device
// copy of their descriptor tables, and the problem list it was built from
struct GraphEntry {
    std::vector<cudaGraphExec_t> execs;
    std::vector<void*> dev_blobs;
    std::vector<unsigned char> problems;
    int64_t kernels = 0;  // kernel launches one replay makes
};

}  // namespace

struct oz2_context {
    cudaStream_t stream = nullptr;
    int device = 0;
    int num_sms = 148;
    size_t ws_limit = 0, resident_hint = 0;
    uint8_t* ws = nullptr;
    size_t ws_size = 0;
    uint64_t ws_gen = 0;
    int* d_err = nullptr;
    std::map<std::pair<int, int64_t>, std::unique_ptr<Plan>> plans;
    int64_t tiling[6] = {0, 0, 0, 0, 0, 0};
    int tuning[3] = {1, 1, 1};
    bool profiling = false;
    std::vector<std::pair<int, cudaEvent_t>> marks;
    std::vector<cudaEvent_t> pool;
    size_t pool_used = 0;
    // pinned staging ring for large descriptor blobs (read by a copy kernel through its device
    // mapping)
    void* ring_host[kRing] = {};
    void* ring_dev[kRing] = {};
    size_t ring_cap[kRing] = {};
    cudaEvent_t ring_ev[kRing] = {};
    bool ring_used[kRing] = {};
    int ring_next = 0;
    // the highest-priority stream for those copies: their few blocks are dispatched ahead of
    // the native tiles' cuBLAS blocks on the other streams
    cudaStream_t xfer = nullptr;
    cudaEvent_t xfer_in = nullptr;
    // pinned buffer that kernels write small results into for the host to read
    void* rb_host = nullptr;
    void* rb_dev = nullptr;
    size_t rb_cap = 0;
    // GEMM configuration: forced by the caller, tuned per problem-set shape, last used
    GemmConfig forced;
    bool has_forced = false;
    std::map<std::string, GemmConfig> tuned;
    GemmConfig last_cfg;
    // CUDA graphs of grouped calls, captured on a private stream (the caller's stream may be
    // the legacy default stream, which cannot be captured) and launched on the caller's stream
    bool graph_mode = false;
    cudaStream_t cap_stream = nullptr;
    std::map<uint64_t, GraphEntry> graphs;
    GraphEntry* capturing = nullptr;  // entry being filled by the current grouped call
    // adaptive s: MLP parameters on the device, second workspace for the per-tile phase
    float* d_mlp = nullptr;
    bool mlp_loaded = false;
    float mlp_threshold = 0.9f;
    int adaptive_tile = 512;
    int probe_kind = 0;  // 0: kProbeCols columns entry by entry, 1: Freivalds, 2: both, 3: none
    uint8_t* ws2 = nullptr;
    size_t ws2_size = 0;
    int64_t astats[kAdaptiveStats] = {};
    int64_t gbytes[3] = {};  // last adaptive call's GEMM: plane bytes read, residue bytes written, tile batches
    cublasHandle_t cublas = nullptr;  // native FP64 GEMM of tiles no moduli set brings to the target
    cudaStream_t cublas_stream = nullptr;
    bool cublas_bound = false;        // cublas_stream is set on the handle
    // native tiles run on their own stream, beside the emulation of the other tiles
    cudaStream_t nat_stream = nullptr;
    cudaEvent_t nat_fork = nullptr, nat_join = nullptr, nat_t0 = nullptr, nat_t1 = nullptr;
    bool nat_pending = false;         // the caller's stream must still wait for nat_join
    double native_ms = 0.0;           // device time of the last call's native tiles (profiling)
    int64_t launches = 0;  // kernels launched through this handle (graph replays included)
    bool capture_ok = true;           // false when part of the call ran outside the graphs
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
#define OZ2_CUDA(h, call)                                      \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, #call); \
    } while (0)

bool op_ok(char t) { return t == 'N' || t == 'n' || t == 'T' || t == 't' || t == 'C' || t == 'c'; }
bool is_n(char t) { return t == 'N' || t == 'n'; }
bool is_c(char t) { return t == 'C' || t == 'c'; }
size_t align256(size_t v) { return (v + 255) & ~size_t{255}; }

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

// plans are cached per (s, k); k is the plan's inner length (2k for complex)
// ext: the adaptive path's range s <= 32 (the extended sets above 24); the reference-facing calls
// keep s <= 24
int get_plan(oz2_context* h, int s, int64_t k, const Plan** out, bool ext = false) {
    if (!ext && s > kMaxModuli) {
        char buf[160];
        return fail(h, OZ2_EINVAL, plan_error_text(s, k, 1, buf, sizeof buf));
    }
    if (ext && (s < 2 || s > kMaxModuliExt))
        return fail(h, OZ2_EINVAL, "oz2: num_moduli must be in [2, " + std::to_string(kMaxModuliExt) + "]");
    auto key = std::make_pair(s, k);
    auto it = h->plans.find(key);
    if (it != h->plans.end()) {
        *out = it->second.get();
        return OZ2_OK;
    }
    auto p = std::make_unique<Plan>();
    const int st = make_plan_ext(s, k, *p);
    if (st) {
        char buf[160];
        plan_error_text(s, k, st, buf, sizeof buf);
        return fail(h, st == 5 ? OZ2_EOVERFLOW : (st == 1 ? OZ2_EINVAL : OZ2_EINTERNAL), buf);
    }
    *out = p.get();
    h->plans.emplace(key, std::move(p));
    return OZ2_OK;
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

void drop_graphs(oz2_context* h) {
    for (auto& kv : h->graphs) {
        for (auto e : kv.second.execs) cudaGraphExecDestroy(e);
        for (auto b : kv.second.dev_blobs) cudaFree(b);
    }
    h->graphs.clear();
    h->capturing = nullptr;
}

int ensure_workspace(oz2_context* h, size_t bytes) {
    if (h->ws_size >= bytes) return OZ2_OK;
    OZ2_CUDA(h, cudaStreamSynchronize(h->stream));
    drop_graphs(h);
    if (h->ws) cudaFree(h->ws);
    h->ws = nullptr;
    h->ws_size = 0;
    ++h->ws_gen;
    if (cudaMalloc(&h->ws, bytes) != cudaSuccess) {
        cudaGetLastError();
        h->ws = nullptr;
        return fail(h, OZ2_ENOMEM, "oz2: workspace allocation failed");
    }
    h->ws_size = bytes;
    return OZ2_OK;
}

// ---------------------------------------------------------------- problem -> tasks -> program
struct Prob {  // one validated problem with m, n, k > 0 and alpha != 0
    char ta, tb;
    int64_t m, n, k;
    double alpha[2], beta[2];
    const double* A;
    int64_t lda;
    const double* B;
    int64_t ldb;
    double* C;
    int64_t ldc;
    int G;  // 1 real, 3 complex (3M)
    const Plan* plan;
};

// bytes of one problem (or one C tile of mb x nb) in the workspace
struct Sizes {
    size_t maxA, maxB, planesA, planesB, resid;
    size_t total() const { return align256(maxA) + align256(maxB) + align256(planesA) + align256(planesB) + align256(resid); }
};
Sizes sizes_for(int64_t m, int64_t n, int64_t k, int s, int G, int64_t mb, int64_t nb) {
    Sizes z;
    z.maxA = static_cast<size_t>(m) * 8;
    z.maxB = static_cast<size_t>(n) * 8;
    z.planesA = static_cast<size_t>(G) * s * plane_geom(mb, k, kGemmIPad).plane_bytes;
    z.planesB = static_cast<size_t>(G) * s * plane_geom(nb, k, kGemmJ).plane_bytes;
    z.resid = static_cast<size_t>(G) * s * nb * round_up(mb, 32);
    return z;
}

SplitItem side_item(const Prob& p, bool a_side, int64_t r0, int64_t rows, unsigned long long* maxbits,
                    int8_t* planes, const ModConst* mc) {
    SplitItem it{};
    const bool cplx = p.G == 3;
    const int w = cplx ? 2 : 1;
    if (a_side) {
        it.row_contig = is_n(p.ta);
        it.X = p.A + w * (it.row_contig ? r0 : r0 * p.lda);
        it.ldx = p.lda;
        it.conj = cplx && is_c(p.ta);
        it.rows_pad = plane_geom(rows, p.k, kGemmIPad).rows_pad;
    } else {
        it.row_contig = !is_n(p.tb);
        it.X = p.B + w * (it.row_contig ? r0 : r0 * p.ldb);
        it.ldx = p.ldb;
        it.conj = cplx && is_c(p.tb);
        it.rows_pad = plane_geom(rows, p.k, kGemmJ).rows_pad;
    }
    it.rows = rows;
    it.k = p.k;
    it.cplx = cplx;
    it.tk = p.plan->tk;
    it.s = p.plan->s;
    it.maxbits = maxbits + r0;
    it.planes = planes;
    it.kb_total = ceil_div(p.k, kTileK);
    it.plane_bytes = it.rows_pad * it.kb_total * kTileK;
    for (int t = 0; t < it.s; ++t) it.mc[t] = mc[t];
    return it;
}

ScaleItem scale_item(const Prob& p, bool a_side, unsigned long long* out) {
    ScaleItem it{};
    const bool cplx = p.G == 3;
    it.X = a_side ? p.A : p.B;
    it.ldx = a_side ? p.lda : p.ldb;
    it.rows = a_side ? p.m : p.n;
    it.k = p.k;
    it.row_contig = a_side ? is_n(p.ta) : !is_n(p.tb);
    it.cplx = cplx;
    it.out = out;
    return it;
}

// one GEMM + CRT unit: C rows [i0, i0+mb) x columns [j0, j0+nb) of a problem
struct Task {
    const Prob* p;
    int64_t i0, j0, mb, nb;
    bool split_a, split_b;
    unsigned long long *maxA, *maxB;  // of the whole problem
    int8_t *planesA, *planesB;
    uint8_t* resid;
    int64_t ldr;
    bool fuse_a = false, fuse_b = false;  // the side's scale pass runs inside its split
};

// whether a side's scale pass is fused into its split (the split kernel then writes its maxima)
bool fuse_side(const Prob& p, bool a_side) {
    return fuse_scale(p.G == 3, a_side ? is_n(p.ta) : !is_n(p.tb), p.k);
}

template <class Item>
void add_grouped(Program& prog, std::vector<Item>& items, Op::Kind kind, int64_t (*geom)(Item&, int64_t),
                 const Plan* plan, bool cplx) {
    int64_t blocks = 0;
    for (auto& it : items) blocks += geom(it, blocks);
    Op op;
    op.kind = kind;
    op.count = static_cast<int>(items.size());
    op.blocks = blocks;
    op.plan = plan;
    op.cplx = cplx;
    op.off = prog.add(items.data(), items.size() * sizeof(Item));
    prog.ops.push_back(op);
}

int64_t split_geom(SplitItem& it, int64_t b0) { return split_geometry(it, b0); }
int64_t crt_geom(CrtItem& it, int64_t b0) { return crt_item_blocks(it, b0); }

// Appends split, GEMM and CRT operations for a list of tasks (launches grouped by kernel variant)
void plan_tasks(Program& prog, const std::vector<Task>& tasks, const GemmConfig& cfg) {
    // split: group by (row_contig, complex / fused scale, limb path: narrow, wide, widest)
    std::map<std::tuple<int, int, int>, std::vector<SplitItem>> split_groups;
    for (const Task& t : tasks) {
        const Prob& p = *t.p;
        const ModConst* mc = p.plan->mc;
        const int wide = p.plan->tk > kWideScaleBits ? 2 : (p.plan->tk > kNarrowScaleBits ? 1 : 0);
        if (t.split_b) {
            SplitItem it = side_item(p, false, t.j0, t.nb, t.maxB, t.planesB, mc);
            it.fuse = t.fuse_b;
            split_groups[{it.row_contig, it.cplx + 2 * it.fuse, wide}].push_back(it);
        }
        if (t.split_a) {
            SplitItem it = side_item(p, true, t.i0, t.mb, t.maxA, t.planesA, mc);
            it.fuse = t.fuse_a;
            split_groups[{it.row_contig, it.cplx + 2 * it.fuse, wide}].push_back(it);
        }
    }
    for (auto& kv : split_groups) add_grouped(prog, kv.second, Op::Split, split_geom, nullptr, false);
    Op mk;
    mk.kind = Op::Mark;
    mk.stage = kSplit;
    prog.ops.push_back(mk);

    // GEMM: one persistent launch over every task; largest work first. Real tasks of s <= 8 with
    // one exact k chunk take the GEMM with the CRT in its epilogue instead (one launch per plan)
    auto crt_in_gemm = [](const Task& t) {
        const Prob& p = *t.p;
        return crt_fusion() && p.G == 1 && p.plan->s <= kCrtFusedMaxS && ceil_div(p.k, kTileK) <= kExactKB;
    };
    std::vector<GemmItem> gi;
    std::map<const Plan*, std::pair<int64_t, std::vector<GemmItem>>> fused;  // plan -> (jobs, items)
    std::vector<size_t> order(tasks.size());
    for (size_t i = 0; i < tasks.size(); ++i) order[i] = i;
    auto work = [&](size_t i) {
        const Task& t = tasks[i];
        return static_cast<double>(t.p->G) * t.p->plan->s * gemm_tiles_i(t.mb, cfg.bn) * ceil_div(t.nb, kGemmJ) *
               ceil_div(t.p->k, kTileK);
    };
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return work(a) > work(b); });
    int64_t jobs = 0;
    for (size_t oi : order) {
        const Task& t = tasks[oi];
        const Prob& p = *t.p;
        const bool fz = crt_in_gemm(t);
        const int bn = fz ? 128 : cfg.bn;
        GemmItem g{};
        g.planes_i = t.planesA;
        g.planes_j = t.planesB;
        g.resid = t.resid;
        g.pstride_i = plane_geom(t.mb, p.k, kGemmIPad).plane_bytes;
        g.pstride_j = plane_geom(t.nb, p.k, kGemmJ).plane_bytes;
        g.rstride = t.nb * t.ldr;
        g.ldr = t.ldr;
        g.m = t.mb;
        g.n = t.nb;
        g.kb_total = ceil_div(p.k, kTileK);
        g.tiles_i = static_cast<int>(gemm_tiles_i(t.mb, bn));
        g.tiles_j = static_cast<int>(ceil_div(t.nb, kGemmJ));
        g.tiles = static_cast<int64_t>(g.tiles_i) * g.tiles_j;
        g.s = p.plan->s;
        g.groups = p.G;
        g.job0 = jobs;
        const ModConst* mc = p.plan->mc;
        for (int q = 0; q < g.s; ++q) {
            g.mod_m[q] = mc[q].m;
            g.mod_mu[q] = mc[q].mu;
            g.mod_kbias[q] = mc[q].kbias;
            g.mod_kbias30[q] = mc[q].kbias30;
            g.mod_mx31[q] = mc[q].mx31;
            g.mod_mxs[q] = mc[q].mxs;
        }
        if (fz) {  // one job per tile; the epilogue writes C
            auto& f = fused[p.plan];
            g.job0 = f.first;
            g.C = p.C + t.i0 + t.j0 * p.ldc;
            g.ldc = p.ldc;
            g.crt_maxA = t.maxA + t.i0;
            g.crt_maxB = t.maxB + t.j0;
            g.crt_tk = p.plan->tk;
            g.crt_alpha = p.alpha[0];
            g.crt_beta = p.beta[0];
            f.first += g.tiles;
            f.second.push_back(g);
            continue;
        }
        jobs += g.tiles * p.G * g.s;
        gi.push_back(g);
    }
    if (!gi.empty()) {
        Op go;
        go.kind = Op::Gemm;
        go.count = static_cast<int>(gi.size());
        go.jobs = jobs;
        go.cfg = cfg;
        go.off = prog.add(gi.data(), gi.size() * sizeof(GemmItem));
        prog.ops.push_back(go);
    }
    for (auto& kv : fused) {
        Op go;
        go.kind = Op::GemmCrt;
        go.count = static_cast<int>(kv.second.second.size());
        go.jobs = kv.second.first;
        go.cfg = cfg;
        go.plan = kv.first;
        go.off = prog.add(kv.second.second.data(), kv.second.second.size() * sizeof(GemmItem));
        prog.ops.push_back(go);
    }
    mk.stage = kGemm;
    prog.ops.push_back(mk);

    // CRT: group by (s, complex); the CRT table of s is a kernel parameter
    std::map<std::pair<int, int>, std::pair<const Plan*, std::vector<CrtItem>>> crt_groups;
    for (const Task& t : tasks) {
        if (crt_in_gemm(t)) continue;
        const Prob& p = *t.p;
        const bool cplx = p.G == 3;
        const int w = cplx ? 2 : 1;
        CrtItem c{};
        c.resid = t.resid;
        c.rstride = t.nb * t.ldr;
        c.gstride = c.rstride * p.plan->s;
        c.ldr = t.ldr;
        c.m = t.mb;
        c.n = t.nb;
        c.ldc = p.ldc;
        c.maxA = t.maxA + t.i0;
        c.maxB = t.maxB + t.j0;
        c.tk = p.plan->tk;
        c.ar = p.alpha[0];
        c.ai = p.alpha[1];
        c.br = p.beta[0];
        c.bi = p.beta[1];
        c.C = p.C + w * (t.i0 + t.j0 * p.ldc);
        c.mma = crt_uses_mma(*p.plan, cplx) ? 1 : 0;
        auto& grp = crt_groups[{p.plan->s, cplx}];
        grp.first = p.plan;
        grp.second.push_back(c);
    }
    for (auto& kv : crt_groups)
        add_grouped(prog, kv.second.second, Op::Crt, crt_geom, kv.second.first, kv.first.second != 0);
    mk.stage = kCrt;
    prog.ops.push_back(mk);
}

void plan_scale(oz2_context* h, Program& prog, std::vector<ScaleItem>& items) {
    // group by (row_contig, complex)
    std::map<std::pair<int, int>, std::vector<ScaleItem>> groups;
    for (auto& it : items) groups[{it.row_contig, it.cplx}].push_back(it);
    for (auto& kv : groups) {
        int64_t blocks = 0;
        for (auto& it : kv.second) blocks += scale_item_blocks(it, h->num_sms, blocks);
        Op op;
        op.kind = Op::Scale;
        op.count = static_cast<int>(kv.second.size());
        op.blocks = blocks;
        op.off = prog.add(kv.second.data(), kv.second.size() * sizeof(ScaleItem));
        prog.ops.push_back(op);
    }
    Op mk;
    mk.kind = Op::Mark;
    mk.stage = kScale;
    prog.ops.push_back(mk);
}

// one-dimensional grids: every launch must stay below 2^31 blocks
int check_grid(oz2_context* h, const Program& prog) {
    for (const Op& op : prog.ops)
        if (op.blocks > 0x7FFFFFFFll) return fail(h, OZ2_EINVAL, "oz2: problem too large for one launch");
    return OZ2_OK;
}

// ---------------------------------------------------------------- issuing a program
// the transfer stream starts after everything issued to the caller's stream so far
int xfer_fork(oz2_context* h) {
    if (!h->xfer) {
        int least = 0, greatest = 0;
        OZ2_CUDA(h, cudaDeviceGetStreamPriorityRange(&least, &greatest));
        OZ2_CUDA(h, cudaStreamCreateWithPriority(&h->xfer, cudaStreamNonBlocking, greatest));
        OZ2_CUDA(h, cudaEventCreateWithFlags(&h->xfer_in, cudaEventDisableTiming));
    }
    OZ2_CUDA(h, cudaEventRecord(h->xfer_in, h->stream));
    OZ2_CUDA(h, cudaStreamWaitEvent(h->xfer, h->xfer_in, 0));
    return OZ2_OK;
}

// copies host bytes to device memory on the stream: small blobs through a kernel parameter,
// large ones through the pinned staging ring and a copy kernel on the transfer stream (no copy
// engine: see launch_sm_copy)
int put_blob(oz2_context* h, const void* data, size_t bytes, unsigned char* dev) {
    if (bytes == 0) return OZ2_OK;
    if (bytes <= kParamBlobBytes) {
        launch_write_blob(data, bytes, dev, h->stream);
        ++h->launches;
        return OZ2_OK;
    }
    const int slot = h->ring_next;
    h->ring_next = (h->ring_next + 1) % kRing;
    if (h->ring_used[slot]) OZ2_CUDA(h, cudaEventSynchronize(h->ring_ev[slot]));
    if (!h->ring_ev[slot]) OZ2_CUDA(h, cudaEventCreateWithFlags(&h->ring_ev[slot], cudaEventDisableTiming));
    if (h->ring_cap[slot] < bytes) {
        // pinned allocations are slow and synchronise: grow in powers of two from 1 MiB, to at
        // least twice this blob, so that the next calls' blobs (which vary with the problem list)
        // rarely grow a slot again
        size_t cap = std::max(h->ring_cap[slot] * 2, size_t{1} << 20);
        while (cap < 2 * bytes) cap *= 2;
        if (h->ring_host[slot]) cudaFreeHost(h->ring_host[slot]);
        h->ring_host[slot] = h->ring_dev[slot] = nullptr;
        h->ring_cap[slot] = 0;
        OZ2_CUDA(h, cudaHostAlloc(&h->ring_host[slot], cap, cudaHostAllocMapped));
        OZ2_CUDA(h, cudaHostGetDevicePointer(&h->ring_dev[slot], h->ring_host[slot], 0));
        h->ring_cap[slot] = cap;
    }
    std::memcpy(h->ring_host[slot], data, bytes);
    if (int st = xfer_fork(h)) return st;  // the region's earlier readers have finished
    launch_sm_copy(h->ring_dev[slot], dev, bytes, h->xfer);
    ++h->launches;
    OZ2_CUDA(h, cudaEventRecord(h->ring_ev[slot], h->xfer));
    OZ2_CUDA(h, cudaStreamWaitEvent(h->stream, h->ring_ev[slot], 0));
    h->ring_used[slot] = true;
    return OZ2_OK;
}

// reads small device arrays into host memory once the stream's work so far has run: a copy
// kernel writes them into mapped pinned memory, the host waits for the stream and copies them
// out (no copy engine: see launch_sm_copy)
struct HostRead {
    void* dst;
    const void* src;
    size_t bytes;
};
int read_back(oz2_context* h, std::initializer_list<HostRead> reads) {
    size_t total = 0;
    for (const HostRead& r : reads) total += (r.bytes + 15) & ~size_t{15};
    if (h->rb_cap < total) {
        OZ2_CUDA(h, cudaStreamSynchronize(h->stream));
        if (h->rb_host) cudaFreeHost(h->rb_host);
        h->rb_host = h->rb_dev = nullptr;
        h->rb_cap = 0;
        size_t cap = size_t{1} << 20;  // pinned allocations are slow: room for twice the request
        while (cap < 2 * total) cap *= 2;
        OZ2_CUDA(h, cudaHostAlloc(&h->rb_host, cap, cudaHostAllocMapped));
        OZ2_CUDA(h, cudaHostGetDevicePointer(&h->rb_dev, h->rb_host, 0));
        h->rb_cap = cap;
    }
    if (int st = xfer_fork(h)) return st;
    size_t off = 0;
    for (const HostRead& r : reads) {
        launch_sm_copy(r.src, static_cast<unsigned char*>(h->rb_dev) + off, r.bytes, h->xfer);
        ++h->launches;
        off += (r.bytes + 15) & ~size_t{15};
    }
    OZ2_CUDA(h, cudaStreamSynchronize(h->xfer));
    off = 0;
    for (const HostRead& r : reads) {
        std::memcpy(r.dst, static_cast<const unsigned char*>(h->rb_host) + off, r.bytes);
        off += (r.bytes + 15) & ~size_t{15};
    }
    return OZ2_OK;
}

int upload(oz2_context* h, const Program& prog, unsigned char* dev) {
    return put_blob(h, prog.blob.data(), prog.blob.size(), dev);
}

void issue(oz2_context* h, const Program& prog, const unsigned char* dev) {
    const unsigned char* hb = prog.blob.data();
    for (const Op& op : prog.ops) {
        if (op.kind != Op::Mark) ++h->launches;
        switch (op.kind) {
            case Op::Memset: launch_fill(op.ptr, 0, op.bytes, h->stream); break;
            case Op::Scale:
                launch_scale(reinterpret_cast<const ScaleItem*>(dev + op.off), reinterpret_cast<const ScaleItem*>(hb + op.off),
                             op.count, op.blocks, h->stream);
                break;
            case Op::Split:
                launch_split(reinterpret_cast<const SplitItem*>(dev + op.off), reinterpret_cast<const SplitItem*>(hb + op.off),
                             op.count, op.blocks, h->d_err, h->stream);
                break;
            case Op::Gemm:
                launch_gemm(reinterpret_cast<const GemmItem*>(dev + op.off), op.count, op.jobs, op.cfg, h->num_sms, h->d_err,
                            h->stream);
                break;
            case Op::GemmCrt:
                launch_gemm_crt(reinterpret_cast<const GemmItem*>(dev + op.off), op.count, op.jobs, *op.plan,
                                op.cfg.group_j, h->num_sms, h->d_err, h->stream);
                break;
            case Op::Slice:
                launch_slice(reinterpret_cast<const SplitItem*>(dev + op.off), reinterpret_cast<const SplitItem*>(hb + op.off),
                             op.count, op.blocks, h->stream);
                break;
            case Op::GemmOz1:
                launch_gemm_oz1(reinterpret_cast<const GemmItem*>(dev + op.off), op.count, op.jobs, op.cfg, h->num_sms,
                                h->d_err, h->stream);
                break;
            case Op::Crt:
                launch_crt(reinterpret_cast<const CrtItem*>(dev + op.off), op.count, op.blocks, *op.plan, op.cplx,
                           h->d_err, h->stream);
                break;
            case Op::ScaleC: launch_scale_c(static_cast<double*>(op.ptr), op.ldc, op.m, op.n, op.beta, op.cplx, h->stream); break;
            case Op::Mark: mark(h, op.stage); break;
        }
    }
}

// ---------------------------------------------------------------- GEMM configuration
GemmConfig heuristic_config(const std::vector<const Prob*>& probs) {
    GemmConfig c;
    // narrow problems waste less padding with 128-row tiles along i
    std::vector<int64_t> ms;
    for (auto* p : probs) ms.push_back(p->m);
    std::sort(ms.begin(), ms.end());
    const int64_t med = ms.empty() ? 0 : ms[ms.size() / 2];
    c.bn = med > 0 && med <= 384 ? 128 : 256;
    c.group_j = 16;
    return c;
}

std::string shape_signature(const std::vector<const Prob*>& probs) {
    std::string s;
    char buf[96];
    for (auto* p : probs) {
        std::snprintf(buf, sizeof buf, "%c%c%lld,%lld,%lld,%d,%d;", p->ta, p->tb, static_cast<long long>(p->m),
                      static_cast<long long>(p->n), static_cast<long long>(p->k), p->plan->s, p->G);
        s += buf;
    }
    return s;
}

GemmConfig config_for(oz2_context* h, const std::vector<const Prob*>& probs) {
    if (h->has_forced) return h->forced;
    auto it = h->tuned.find(shape_signature(probs));
    if (it != h->tuned.end()) return it->second;
    return heuristic_config(probs);
}

// ---------------------------------------------------------------- one emulated GEMM (tiled)
struct Layout {
    int64_t mb, nb, pm, pn, kchunks;
    size_t bytes;
};

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

size_t desc_bytes_single(int64_t pm, int64_t pn) {
    const int64_t tiles = pm * pn;
    return 4096 + static_cast<size_t>(2 * tiles) * (sizeof(SplitItem) + 256) +
           static_cast<size_t>(tiles) * (sizeof(GemmItem) + sizeof(CrtItem) + 512) + 2 * sizeof(ScaleItem);
}

// Largest column tile that fits for each row-tile candidate, scored by an analytic time model
// of this implementation (tensor work on padded tiles, HBM traffic of split and CRT, launches).
int choose_layout(oz2_context* h, int64_t m, int64_t n, int64_t k, int s, int G, Layout& out) {
    // a problem whose untiled layout fits the current workspace needs no free-memory query
    const size_t untiled = sizes_for(m, n, k, s, G, m, n).total() + align256(desc_bytes_single(1, 1));
    const size_t limit =
        untiled <= h->ws_size && (!h->ws_limit || untiled <= h->ws_limit) ? untiled : budget(h);
    double best = std::numeric_limits<double>::infinity();
    const bool pow2 = h->tuning[2] != 0;
    const auto nbs = tile_candidates(n, kGemmJ, pow2);
    for (int64_t mb : tile_candidates(m, kGemmIPad, pow2)) {
        for (int64_t nb : nbs) {
            const int64_t pm = ceil_div(m, mb), pn = ceil_div(n, nb);
            const size_t bytes = sizes_for(m, n, k, s, G, mb, nb).total() + align256(desc_bytes_single(pm, pn));
            if (bytes > limit) continue;
            const double gemm = 2.0 * G * s * k * static_cast<double>(pm * round_up(mb, kGemmIPad)) *
                                static_cast<double>(pn * round_up(nb, kGemmJ)) / 3.0e15;
            const double split = G * (8.0 + s) * (static_cast<double>(k) * m * (pm > 1 ? pn : 1) +
                                                  static_cast<double>(k) * n) / 5.0e12;
            const double crt = G * (s + 16.0) * static_cast<double>(m) * n / 5.0e12;
            const double t = gemm + split + crt + pm * pn * 4 * 5e-6;
            if (t < best) {
                best = t;
                out = Layout{mb, nb, pm, pn, ceil_div(ceil_div(k, kTileK), kChunkKB), bytes};
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

int run_single(oz2_context* h, const Prob& p) {
    const int s = p.plan->s;
    Layout L;
    int st = choose_layout(h, p.m, p.n, p.k, s, p.G, L);
    if (st) return st;
    if ((st = ensure_workspace(h, L.bytes))) return st;
    h->tiling[0] = L.mb;
    h->tiling[1] = L.nb;
    h->tiling[2] = L.pm;
    h->tiling[3] = L.pn;
    h->tiling[4] = L.kchunks;
    h->tiling[5] = static_cast<int64_t>(L.bytes);
    const Sizes z = sizes_for(p.m, p.n, p.k, s, p.G, L.mb, L.nb);
    size_t off = 0;
    auto carve = [&](size_t b) {
        const size_t o = off;
        off += align256(b);
        return h->ws + o;
    };
    auto* maxA = reinterpret_cast<unsigned long long*>(carve(z.maxA));
    auto* maxB = reinterpret_cast<unsigned long long*>(carve(z.maxB));
    auto* planesA = reinterpret_cast<int8_t*>(carve(z.planesA));
    auto* planesB = reinterpret_cast<int8_t*>(carve(z.planesB));
    auto* resid = carve(z.resid);
    unsigned char* dev_desc = carve(0);

    const std::vector<const Prob*> probs{&p};
    const GemmConfig cfg = config_for(h, probs);
    h->last_cfg = cfg;
    Program prog;
    Op mk;
    mk.kind = Op::Mark;
    mk.stage = kBegin;
    prog.ops.push_back(mk);
    Op ms;
    ms.kind = Op::Memset;
    ms.ptr = maxA;
    ms.bytes = reinterpret_cast<unsigned char*>(planesA) - reinterpret_cast<unsigned char*>(maxA);
    prog.ops.push_back(ms);
    const bool fa = fuse_side(p, true), fb = fuse_side(p, false);
    std::vector<ScaleItem> sc;
    if (!fa) sc.push_back(scale_item(p, true, maxA));
    if (!fb) sc.push_back(scale_item(p, false, maxB));
    plan_scale(h, prog, sc);
    const int64_t ldr = round_up(L.mb, 32);
    for (int64_t j0 = 0; j0 < p.n; j0 += L.nb) {
        for (int64_t i0 = 0; i0 < p.m; i0 += L.mb) {
            Task t{&p, i0, j0, std::min(L.mb, p.m - i0), std::min(L.nb, p.n - j0), L.pm > 1 || j0 == 0, i0 == 0,
                   maxA, maxB, planesA, planesB, resid, ldr, fa, fb};
            plan_tasks(prog, {t}, cfg);
        }
    }
    if (prog.blob.size() > align256(desc_bytes_single(L.pm, L.pn)))
        return fail(h, OZ2_EINTERNAL, "oz2: descriptor region too small");
    if ((st = check_grid(h, prog))) return st;
    if ((st = upload(h, prog, dev_desc))) return st;
    issue(h, prog, dev_desc);
    return OZ2_OK;
}

// ---------------------------------------------------------------- grouped
int run_grouped(oz2_context* h, std::vector<Prob>& probs) {
    // every problem untiled; batches of problems whose workspace fits the budget
    const size_t limit = budget(h);
    std::vector<std::vector<size_t>> batches;
    std::vector<size_t> cur;
    size_t cur_bytes = 4096;
    std::vector<size_t> need(probs.size());
    for (size_t i = 0; i < probs.size(); ++i) {
        const Prob& p = probs[i];
        need[i] = sizes_for(p.m, p.n, p.k, p.plan->s, p.G, p.m, p.n).total() + 4 * sizeof(SplitItem) + 2048;
        if (need[i] + 4096 > limit) {  // alone too large: the tiled single path
            h->capture_ok = false;
            int st = run_single(h, p);
            if (st) return st;
            continue;
        }
        if (cur_bytes + need[i] > limit && !cur.empty()) {
            batches.push_back(cur);
            cur.clear();
            cur_bytes = 4096;
        }
        cur.push_back(i);
        cur_bytes += need[i];
    }
    if (!cur.empty()) batches.push_back(cur);

    size_t max_bytes = 0;
    for (auto& b : batches) {
        size_t sum = 4096;
        for (size_t i : b) sum += need[i];
        max_bytes = std::max(max_bytes, sum);
    }
    int st = ensure_workspace(h, max_bytes);
    if (st) return st;

    for (auto& b : batches) {
        std::vector<const Prob*> bp;
        for (size_t i : b) bp.push_back(&probs[i]);
        const GemmConfig cfg = config_for(h, bp);
        h->last_cfg = cfg;
        // carve: maxima of all problems first (one memset), then planes and residues
        size_t off = 0;
        auto carve = [&](size_t bytes) {
            const size_t o = off;
            off += align256(bytes);
            return h->ws + o;
        };
        std::vector<Task> tasks;
        std::vector<ScaleItem> sc;
        std::vector<std::pair<unsigned long long*, unsigned long long*>> mx;
        for (const Prob* p : bp)
            mx.emplace_back(reinterpret_cast<unsigned long long*>(carve(p->m * 8)),
                            reinterpret_cast<unsigned long long*>(carve(p->n * 8)));
        const size_t max_end = off;
        for (size_t q = 0; q < bp.size(); ++q) {
            const Prob& p = *bp[q];
            const Sizes z = sizes_for(p.m, p.n, p.k, p.plan->s, p.G, p.m, p.n);
            auto* pa = reinterpret_cast<int8_t*>(carve(z.planesA));
            auto* pb = reinterpret_cast<int8_t*>(carve(z.planesB));
            auto* rs = carve(z.resid);
            const bool fa = fuse_side(p, true), fb = fuse_side(p, false);
            tasks.push_back(Task{&p, 0, 0, p.m, p.n, true, true, mx[q].first, mx[q].second, pa, pb, rs,
                                 round_up(p.m, 32), fa, fb});
            if (!fa) sc.push_back(scale_item(p, true, mx[q].first));
            if (!fb) sc.push_back(scale_item(p, false, mx[q].second));
        }
        unsigned char* dev_desc = carve(0);
        Program prog;
        Op mk;
        mk.kind = Op::Mark;
        mk.stage = kBegin;
        prog.ops.push_back(mk);
        Op ms;
        ms.kind = Op::Memset;
        ms.ptr = h->ws;
        ms.bytes = max_end;
        prog.ops.push_back(ms);
        plan_scale(h, prog, sc);
        plan_tasks(prog, tasks, cfg);
        if (static_cast<size_t>(dev_desc - h->ws) + prog.blob.size() > h->ws_size)
            return fail(h, OZ2_EINTERNAL, "oz2: descriptor region too small");
        if ((st = check_grid(h, prog))) return st;

        if (h->capturing) {
            void* dev_blob = nullptr;
            OZ2_CUDA(h, cudaMalloc(&dev_blob, std::max<size_t>(prog.blob.size(), 256)));
            h->capturing->dev_blobs.push_back(dev_blob);
            OZ2_CUDA(h, cudaMemcpy(dev_blob, prog.blob.data(), prog.blob.size(), cudaMemcpyHostToDevice));
            cudaGraph_t g;
            if (!h->cap_stream) OZ2_CUDA(h, cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking));
            const bool prof = h->profiling;
            cudaStream_t user = h->stream;
            h->profiling = false;  // no event records inside a graph
            h->stream = h->cap_stream;
            cudaError_t ce = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
            if (ce == cudaSuccess) {
                const int64_t before = h->launches;
                issue(h, prog, static_cast<unsigned char*>(dev_blob));
                h->capturing->kernels += h->launches - before;
                ce = cudaStreamEndCapture(h->stream, &g);
            }
            h->stream = user;
            h->profiling = prof;
            if (ce != cudaSuccess) return cuda_fail(h, ce, "cudaStreamEndCapture");
            cudaGraphExec_t exec = nullptr;
            const cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
            cudaGraphDestroy(g);
            if (ie != cudaSuccess) return cuda_fail(h, ie, "cudaGraphInstantiate");
            h->capturing->execs.push_back(exec);
            OZ2_CUDA(h, cudaGraphLaunch(exec, h->stream));
        } else {
            if ((st = upload(h, prog, dev_desc))) return st;
            issue(h, prog, dev_desc);
        }
    }
    h->tiling[0] = h->tiling[1] = h->tiling[2] = h->tiling[3] = h->tiling[4] = 0;
    h->tiling[5] = static_cast<int64_t>(max_bytes);
    return OZ2_OK;
}


// ---------------------------------------------------------------- adaptive s per tile
int ensure_ws2(oz2_context* h, size_t bytes) {
    if (h->ws2_size >= bytes) return OZ2_OK;
    OZ2_CUDA(h, cudaStreamSynchronize(h->stream));
    drop_graphs(h);
    if (h->ws2) cudaFree(h->ws2);
    h->ws2 = nullptr;
    h->ws2_size = 0;
    // tile batches vary from call to call: a quarter of headroom saves most regrowths
    const size_t grown = bytes + bytes / 4;
    if (cudaMalloc(&h->ws2, grown) == cudaSuccess) {
        h->ws2_size = grown;
        return OZ2_OK;
    }
    cudaGetLastError();
    if (cudaMalloc(&h->ws2, bytes) != cudaSuccess) {
        cudaGetLastError();
        return fail(h, OZ2_ENOMEM, "oz2: workspace allocation failed");
    }
    h->ws2_size = bytes;
    return OZ2_OK;
}

// the handle's cuBLAS handle, created on first use and bound to stream st
int cublas_on(oz2_context* h, cudaStream_t st) {
    if (!h->cublas) {
        if (cublasCreate(&h->cublas) != CUBLAS_STATUS_SUCCESS) {
            h->cublas = nullptr;
            return fail(h, OZ2_ECUDA, "oz2: cublasCreate failed");
        }
        cublasSetMathMode(h->cublas, CUBLAS_DEFAULT_MATH);
        h->cublas_bound = false;
    }
    // setting the stream resets cuBLAS's workspace: only when the stream changed
    if (!h->cublas_bound || h->cublas_stream != st) {
        if (cublasSetStream(h->cublas, st) != CUBLAS_STATUS_SUCCESS)
            return fail(h, OZ2_ECUDA, "oz2: cublasSetStream failed");
        h->cublas_stream = st;
        h->cublas_bound = true;
    }
    return OZ2_OK;
}

// C[i0:i0+mb, j0:j0+nb] = alpha op(A) op(B) + beta C in native FP64 (cuBLAS DGEMM, default math:
// no emulation), for tiles whose inputs span more exponent range than 32 moduli cover
int native_gemm(oz2_context* h, cudaStream_t st, const Prob& p, int64_t i0, int64_t j0, int64_t mb, int64_t nb) {
    const int sb = cublas_on(h, st);
    if (sb) return sb;
    const double* A = p.A + (is_n(p.ta) ? i0 : i0 * p.lda);
    const double* B = p.B + (is_n(p.tb) ? j0 * p.ldb : j0);
    double* C = p.C + i0 + j0 * p.ldc;
    const double al = p.alpha[0], be = p.beta[0];
    const cublasStatus_t cs = cublasDgemm_64(h->cublas, is_n(p.ta) ? CUBLAS_OP_N : CUBLAS_OP_T,
                                             is_n(p.tb) ? CUBLAS_OP_N : CUBLAS_OP_T, mb, nb, p.k, &al, A, p.lda, B,
                                             p.ldb, &be, C, p.ldc);
    if (cs != CUBLAS_STATUS_SUCCESS) return fail(h, OZ2_ECUDA, "oz2: native FP64 GEMM failed");
    ++h->launches;
    return OZ2_OK;
}

// `count` tiles of one row of tiles in native FP64, side by side: C[i0:i0+mb, j0 + b nb ...] for
// b < count, one strided batched cuBLAS DGEMM (op(A)'s rows shared, op(B)'s columns and C advance
// by nb per tile). One 512 x 512 tile alone fills well under half of the SMs; a row of them fills
// them all.
int native_gemm_row(oz2_context* h, cudaStream_t st, const Prob& p, int64_t i0, int64_t j0, int64_t mb, int64_t nb,
                    int64_t count) {
    const int sb = cublas_on(h, st);
    if (sb) return sb;
    const double* A = p.A + (is_n(p.ta) ? i0 : i0 * p.lda);
    const double* B = p.B + (is_n(p.tb) ? j0 * p.ldb : j0);
    double* C = p.C + i0 + j0 * p.ldc;
    const double al = p.alpha[0], be = p.beta[0];
    const cublasStatus_t cs = cublasDgemmStridedBatched_64(
        h->cublas, is_n(p.ta) ? CUBLAS_OP_N : CUBLAS_OP_T, is_n(p.tb) ? CUBLAS_OP_N : CUBLAS_OP_T, mb, nb, p.k, &al, A,
        p.lda, 0, B, p.ldb, is_n(p.tb) ? nb * p.ldb : nb, &be, C, p.ldc, nb * p.ldc, count);
    if (cs != CUBLAS_STATUS_SUCCESS) return fail(h, OZ2_ECUDA, "oz2: native FP64 GEMM failed");
    ++h->launches;
    return OZ2_OK;
}

// opens the native stream's part of a call: it starts after everything issued so far
int native_fork(oz2_context* h) {
    if (!h->nat_stream) {
        OZ2_CUDA(h, cudaStreamCreateWithFlags(&h->nat_stream, cudaStreamNonBlocking));
        OZ2_CUDA(h, cudaEventCreateWithFlags(&h->nat_fork, cudaEventDisableTiming));
        OZ2_CUDA(h, cudaEventCreateWithFlags(&h->nat_join, cudaEventDisableTiming));
        OZ2_CUDA(h, cudaEventCreate(&h->nat_t0));
        OZ2_CUDA(h, cudaEventCreate(&h->nat_t1));
    }
    OZ2_CUDA(h, cudaEventRecord(h->nat_fork, h->stream));
    OZ2_CUDA(h, cudaStreamWaitEvent(h->nat_stream, h->nat_fork, 0));
    return OZ2_OK;
}

// the caller's stream waits for the native tiles
int native_join(oz2_context* h) {
    if (!h->nat_pending) return OZ2_OK;
    h->nat_pending = false;
    OZ2_CUDA(h, cudaEventRecord(h->nat_join, h->nat_stream));
    OZ2_CUDA(h, cudaStreamWaitEvent(h->stream, h->nat_join, 0));
    return OZ2_OK;
}

// tk[s] for one k (0 where s is too small)
void tk_table(int64_t k, int* tk) {
    for (int s = 0; s <= kMaxModuliExt; ++s) tk[s] = s >= 2 ? plan_tk(s, k) : 0;
}

struct TileRef {
    int prob;      // index into the problem list
    int64_t i0, j0, mb, nb;
    int ia, jb;    // panel indices
};

// The certified s of every tile (oz2_certify.cu): per group of problems that fits the budget,
// bf16 planes of the scaled magnitudes and the row / column sums, one persistent tcgen05 GEMM
// launch over all the group's problems whose epilogue keeps two maxima per tile, then one thread
// per tile. A problem with k above one GEMM chunk, or whose planes exceed the budget on their
// own, keeps kNativeS (no certificate: its tiles take the analytic s).
int certify_tiles(oz2_context* h, const std::vector<Prob>& base, const std::vector<TileRef>& tiles, int64_t T,
                  const std::function<unsigned long long*(int)>& maxA, const std::function<unsigned long long*(int)>& maxB,
                  const std::map<int64_t, std::vector<int>>& tk_cache, const std::vector<char>& want, int target_bits,
                  unsigned int* d_q, int* d_sc) {
    const size_t budget = h->ws_limit ? h->ws_limit / 2 : (size_t{4} << 30);
    std::vector<int64_t> first_tile(base.size(), -1), ntile(base.size(), 0);
    for (int64_t t = 0; t < static_cast<int64_t>(tiles.size()); ++t) {
        const int q = tiles[t].prob;
        if (first_tile[q] < 0) first_tile[q] = t;
        ++ntile[q];
    }
    auto bytes_of = [&](const Prob& p) {
        return align256(plane_geom(p.m, 2 * p.k, kGemmIPad).plane_bytes) +
               align256(plane_geom(p.n, 2 * p.k, kGemmJ).plane_bytes) + align256(8 * static_cast<size_t>(p.m)) +
               align256(8 * static_cast<size_t>(p.n));
    };
    size_t q0 = 0;
    while (q0 < base.size()) {
        std::vector<size_t> group;
        size_t q1 = q0, total = 0;
        for (; q1 < base.size(); ++q1) {
            const Prob& p = base[q1];
            if (!want[q1] || p.k > kCertMaxK || bytes_of(p) > budget) continue;  // no certificate for this one
            if (!group.empty() && total + bytes_of(p) > budget) break;
            total += bytes_of(p);
            group.push_back(q1);
        }
        q0 = q1;
        if (group.empty()) continue;
        struct Buf {
            size_t pa, pb, ra, sb;
            PlaneGeom ga, gb;
        };
        std::vector<Buf> buf(group.size());
        size_t off = 0;
        auto carve = [&](size_t b) {
            const size_t o = off;
            off += align256(b);
            return o;
        };
        int64_t nt = 0;
        for (size_t g = 0; g < group.size(); ++g) {
            const Prob& p = base[group[g]];
            Buf& b = buf[g];
            b.ga = plane_geom(p.m, 2 * p.k, kGemmIPad);
            b.gb = plane_geom(p.n, 2 * p.k, kGemmJ);
            b.pa = carve(b.ga.plane_bytes);
            b.pb = carve(b.gb.plane_bytes);
            b.ra = carve(8 * static_cast<size_t>(p.m));
            b.sb = carve(8 * static_cast<size_t>(p.n));
            nt += ntile[group[g]];
        }
        const size_t odesc = off;
        const size_t desc = 2 * align256(2 * group.size() * sizeof(CertPrepItem)) +
                            align256(group.size() * sizeof(GemmItem)) + align256(nt * sizeof(CertTileItem));
        int st = ensure_ws2(h, odesc + desc + 4096);
        if (st) return st;
        unsigned char* w = h->ws2;
        size_t dpos = odesc;
        // bf16 planes of the scaled magnitudes and the sums, grouped by layout
        std::vector<CertPrepItem> prep[2];
        for (size_t g = 0; g < group.size(); ++g) {
            const int q = static_cast<int>(group[g]);
            const Prob& p = base[q];
            const Buf& b = buf[g];
            for (int side = 0; side < 2; ++side) {
                CertPrepItem it{};
                it.X = side ? p.B : p.A;
                it.ldx = side ? p.ldb : p.lda;
                it.rows = side ? p.n : p.m;
                it.k = p.k;
                it.row_contig = side ? !is_n(p.tb) : is_n(p.ta);
                it.maxbits = side ? maxB(q) : maxA(q);
                it.planes = reinterpret_cast<uint8_t*>(w + (side ? b.pb : b.pa));
                it.rows_pad = side ? b.gb.rows_pad : b.ga.rows_pad;
                it.kb_total = b.ga.kb_total;
                it.rsum = reinterpret_cast<double*>(w + (side ? b.sb : b.ra));
                prep[it.row_contig].push_back(it);
            }
        }
        for (int lay = 0; lay < 2; ++lay) {
            if (prep[lay].empty()) continue;
            int64_t blocks = 0;
            for (auto& it : prep[lay]) blocks += cert_prep_blocks(it, blocks);
            unsigned char* dd = w + dpos;
            const size_t nbytes = prep[lay].size() * sizeof(CertPrepItem);
            if ((st = put_blob(h, prep[lay].data(), nbytes, dd))) return st;
            launch_cert_prep(reinterpret_cast<const CertPrepItem*>(dd), prep[lay].data(),
                             static_cast<int>(prep[lay].size()), blocks, h->stream);
            ++h->launches;
            dpos += align256(nbytes);
        }
        // the GEMM over all problems of the group: one job per (256 x 128) tile, s = 1
        std::vector<GemmItem> gi(group.size());
        int64_t jobs = 0;
        for (size_t g = 0; g < group.size(); ++g) {
            const int q = static_cast<int>(group[g]);
            const Prob& p = base[q];
            const Buf& b = buf[g];
            GemmItem& it = gi[g];
            it = GemmItem{};
            it.planes_i = reinterpret_cast<const int8_t*>(w + b.pa);
            it.planes_j = reinterpret_cast<const int8_t*>(w + b.pb);
            it.m = p.m;
            it.n = p.n;
            it.kb_total = b.ga.kb_total;
            it.tiles_i = static_cast<int>(gemm_tiles_i(p.m, 256));
            it.tiles_j = static_cast<int>(ceil_div(p.n, kGemmJ));
            it.tiles = static_cast<int64_t>(it.tiles_i) * it.tiles_j;
            it.s = 1;
            it.groups = 1;
            it.job0 = jobs;
            it.cert_ra = reinterpret_cast<const double*>(w + b.ra);
            it.cert_sb = reinterpret_cast<const double*>(w + b.sb);
            it.cert_q = d_q + 2 * first_tile[q];
            it.cert_tile = T;
            it.cert_na = ceil_div(p.m, T);
            jobs += it.tiles;
        }
        unsigned char* dg = w + dpos;
        if ((st = put_blob(h, gi.data(), gi.size() * sizeof(GemmItem), dg))) return st;
        dpos += align256(gi.size() * sizeof(GemmItem));
        launch_gemm_cert(reinterpret_cast<const GemmItem*>(dg), static_cast<int>(gi.size()), jobs, h->num_sms,
                         h->d_err, h->stream);
        ++h->launches;
        // s per tile
        std::vector<CertTileItem> ti;
        ti.reserve(nt);
        for (size_t g = 0; g < group.size(); ++g) {
            const int q = static_cast<int>(group[g]);
            const Prob& p = base[q];
            const std::vector<int>& tk = tk_cache.at(p.k);
            for (int64_t t = first_tile[q]; t < first_tile[q] + ntile[q]; ++t) {
                const TileRef& r = tiles[t];
                CertTileItem it{};
                it.q = d_q + 2 * t;
                it.maxa = maxA(q) + r.i0;
                it.maxb = maxB(q) + r.j0;
                it.mb = r.mb;
                it.nb = r.nb;
                it.k = p.k;
                it.target_bits = target_bits;
                for (int s = 0; s <= kMaxModuliExt; ++s) it.tk[s] = tk[s];
                it.s_out = d_sc + t;
                ti.push_back(it);
            }
        }
        unsigned char* dt = w + dpos;
        if ((st = put_blob(h, ti.data(), ti.size() * sizeof(CertTileItem), dt))) return st;
        launch_cert_tiles(reinterpret_cast<const CertTileItem*>(dt), static_cast<int>(ti.size()), h->stream);
        ++h->launches;
    }
    return OZ2_OK;
}

// mode: 0 MLP per tile for tiles without a certificate (arbiter cap, probe, rerun at the arbiter's s;
// certified tiles take the arbiter's s), 1 analytic per tile,
// 2 analytic per problem (the largest of its tiles), 3 the problems' own num_moduli, 4 certified
// per tile, 5 certified per problem. The arbiter of a tile is the smaller of its analytic and
// certified s (modes 0, 4, 5; the analytic s alone in modes 1 and 2).
int run_adaptive(oz2_context* h, std::vector<Prob>& base, const std::vector<int>& fixed_s, int target_bits,
                 int mode, float* feat_out = nullptr, int* sa_out = nullptr, int64_t* ntiles_out = nullptr) {
    const int64_t T = h->adaptive_tile;
    for (int q = 0; q < kAdaptiveStats; ++q) h->astats[q] = 0;
    for (int64_t& g : h->gbytes) g = 0;
    // ---- phase 1: maxima, panel statistics, tile features, analytic s, MLP
    std::vector<TileRef> tiles;
    std::vector<int64_t> pa0(base.size()), pb0(base.size());
    int64_t npanels = 0;
    for (size_t q = 0; q < base.size(); ++q) {
        const Prob& p = base[q];
        const int64_t na = ceil_div(p.m, T), nbp = ceil_div(p.n, T);
        pa0[q] = npanels;
        npanels += na;
        pb0[q] = npanels;
        npanels += nbp;
        for (int64_t J = 0; J < nbp; ++J)
            for (int64_t I = 0; I < na; ++I)
                tiles.push_back(TileRef{static_cast<int>(q), I * T, J * T, std::min(T, p.m - I * T),
                                        std::min(T, p.n - J * T), static_cast<int>(pa0[q] + I),
                                        static_cast<int>(pb0[q] + J)});
    }
    const int64_t ntiles = static_cast<int64_t>(tiles.size());
    size_t off = 0;
    auto carve1 = [&](size_t bytes) {
        const size_t o = off;
        off += align256(bytes);
        return o;
    };
    std::vector<size_t> omaxA(base.size()), omaxB(base.size());
    for (size_t q = 0; q < base.size(); ++q) {
        omaxA[q] = carve1(base[q].m * 8);
        omaxB[q] = carve1(base[q].n * 8);
    }
    const size_t ohist = carve1(static_cast<size_t>(npanels) * (kGapBins + 1) * 4);
    const size_t ofail = carve1(static_cast<size_t>(ntiles) * 4);
    const size_t ocq = carve1(static_cast<size_t>(ntiles) * 8);  // the certificate's two maxima per tile
    const size_t zero_end = off;
    const size_t ofeat = carve1(static_cast<size_t>(ntiles) * kFeatures * 4);
    const size_t osa = carve1(static_cast<size_t>(ntiles) * 4);
    const size_t osm = carve1(static_cast<size_t>(ntiles) * 4);
    const size_t osc = carve1(static_cast<size_t>(ntiles) * 4);
    const size_t desc_bytes = 1024 + base.size() * 2 * sizeof(ScaleItem) + npanels * sizeof(StatItem) +
                              ntiles * (sizeof(FeatureItem) + sizeof(ProbeItem) + 2 * sizeof(FreivaldsItem)) +
                              16 * 256;
    const size_t odesc = carve1(desc_bytes);
    // a quarter of headroom: the phase-1 data grows with the tile count, which varies from call to
    // call, and each regrowth drains the stream and reallocates
    int st = h->ws_size >= off ? OZ2_OK : ensure_workspace(h, off + off / 4);
    if (st) return st;
    auto* ws = h->ws;
    auto maxA = [&](int q) { return reinterpret_cast<unsigned long long*>(ws + omaxA[q]); };
    auto maxB = [&](int q) { return reinterpret_cast<unsigned long long*>(ws + omaxB[q]); };
    auto hist = [&](int64_t panel) { return reinterpret_cast<unsigned int*>(ws + ohist) + panel * (kGapBins + 1); };
    int* d_fail = reinterpret_cast<int*>(ws + ofail);
    float* d_feat = reinterpret_cast<float*>(ws + ofeat);
    int* d_sa = reinterpret_cast<int*>(ws + osa);
    int* d_sm = reinterpret_cast<int*>(ws + osm);
    int* d_sc = reinterpret_cast<int*>(ws + osc);
    unsigned int* d_q = reinterpret_cast<unsigned int*>(ws + ocq);
    launch_fill(ws, 0, zero_end, h->stream);
    ++h->launches;

    Program ph1;
    // with every k up to kFusedStatsMaxK one launch per layout takes the row maxima and the panel
    // statistics together (one read of A and B from DRAM); otherwise the scale pass runs first
    int64_t kmax = 0;
    for (const Prob& p : base) kmax = std::max(kmax, p.k);
    const bool fused_stats = kmax <= kFusedStatsMaxK;
    std::vector<ScaleItem> sc;
    for (size_t q = 0; q < base.size() && !fused_stats; ++q) {
        sc.push_back(scale_item(base[q], true, maxA(static_cast<int>(q))));
        sc.push_back(scale_item(base[q], false, maxB(static_cast<int>(q))));
    }
    plan_scale(h, ph1, sc);
    // panel statistics, grouped by layout
    std::map<int, std::vector<StatItem>> stat_groups;
    for (size_t q = 0; q < base.size(); ++q) {
        const Prob& p = base[q];
        for (int side = 0; side < 2; ++side) {
            const int64_t rows = side ? p.n : p.m;
            const bool rowc = side ? !is_n(p.tb) : is_n(p.ta);
            const double* X = side ? p.B : p.A;
            const int64_t ldx = side ? p.ldb : p.lda;
            for (int64_t r0 = 0, pi = 0; r0 < rows; r0 += T, ++pi) {
                StatItem it{};
                it.X = X + (rowc ? r0 : r0 * ldx);
                it.ldx = ldx;
                it.rows = std::min(T, rows - r0);
                it.k = p.k;
                it.row_contig = rowc;
                it.maxbits = (side ? maxB(static_cast<int>(q)) : maxA(static_cast<int>(q))) + r0;
                it.hist = hist((side ? pb0[q] : pa0[q]) + pi);
                stat_groups[rowc].push_back(it);
            }
        }
    }
    struct StatOp {
        size_t off;
        int count;
        int64_t blocks;
    };
    std::vector<StatOp> stat_ops;
    for (auto& kv : stat_groups) {
        int64_t blocks = 0;
        for (auto& it : kv.second)
            blocks += fused_stats ? scale_stat_item_blocks(it, blocks) : stat_item_blocks(it, blocks);
        stat_ops.push_back({ph1.add(kv.second.data(), kv.second.size() * sizeof(StatItem)),
                            static_cast<int>(kv.second.size()), blocks});
    }
    std::vector<FeatureItem> fi(ntiles);
    std::map<int64_t, std::vector<int>> tk_cache;
    for (int64_t t = 0; t < ntiles; ++t) {
        const TileRef& r = tiles[t];
        const Prob& p = base[r.prob];
        FeatureItem& f = fi[t];
        f.hist_a = hist(r.ia);
        f.hist_b = hist(r.jb);
        f.maxbits_a = maxA(r.prob) + r.i0;
        f.maxbits_b = maxB(r.prob) + r.j0;
        f.rows_a = r.mb;
        f.rows_b = r.nb;
        f.k = p.k;
        f.target_bits = target_bits;
        auto it = tk_cache.find(p.k);
        if (it == tk_cache.end()) {
            std::vector<int> tk(kMaxModuliExt + 1);
            tk_table(p.k, tk.data());
            it = tk_cache.emplace(p.k, tk).first;
        }
        for (int s = 0; s <= kMaxModuliExt; ++s) f.tk[s] = it->second[s];
    }
    const size_t ofi = ph1.add(fi.data(), fi.size() * sizeof(FeatureItem));
    if (ph1.blob.size() > desc_bytes) return fail(h, OZ2_EINTERNAL, "oz2: descriptor region too small");
    unsigned char* dd = ws + odesc;
    if ((st = put_blob(h, ph1.blob.data(), ph1.blob.size(), dd))) return st;
    mark(h, kBegin);
    issue(h, ph1, dd);  // scale (its mark closes the scale stage)
    for (const StatOp& so : stat_ops) {
        const StatItem* d_items = reinterpret_cast<const StatItem*>(dd + so.off);
        const StatItem* h_items = reinterpret_cast<const StatItem*>(ph1.blob.data() + so.off);
        if (fused_stats) launch_scale_stats(d_items, h_items, so.count, so.blocks, h->stream);
        else launch_panel_stats(d_items, h_items, so.count, so.blocks, h->stream);
        ++h->launches;
    }
    launch_tile_features(reinterpret_cast<const FeatureItem*>(dd + ofi), static_cast<int>(ntiles), d_feat, d_sa,
                         h->stream);
    const bool use_mlp = mode == 0 && h->mlp_loaded;
    ++h->launches;
    if (use_mlp) {
        launch_mlp_infer(h->d_mlp, static_cast<int>(ntiles), d_feat, h->mlp_threshold, d_sm, nullptr, h->stream);
        ++h->launches;
    }
    constexpr int kNoCertificate = 0x7F7F7F7F;  // the device's fill byte 0x7F: above every s
    std::vector<int> s_an(ntiles), s_ml(ntiles, kMaxModuli), s_ce(ntiles, kNoCertificate);
    const size_t tile_bytes = static_cast<size_t>(ntiles) * 4;
    if (use_mlp) st = read_back(h, {{s_an.data(), d_sa, tile_bytes}, {s_ml.data(), d_sm, tile_bytes}});
    else st = read_back(h, {{s_an.data(), d_sa, tile_bytes}});
    if (st) return st;
    // The certificate costs about three moduli of emulation over the problem and saves about four
    // where the analytic s is emulated, far more where it is native: it runs for the problems
    // with a tile at kCertFromS or above.
    constexpr int kCertFromS = 23;
    const bool certify = mode == 0 || mode == 4 || mode == 5;
    if (certify && mode >= 0) {
        std::vector<char> want(base.size(), 0);
        bool any = false;
        for (int64_t t = 0; t < ntiles; ++t)
            if (s_an[t] >= kCertFromS) any = want[tiles[t].prob] = 1;
        if (any) {
            launch_fill(d_sc, 0x7F, ntiles * 4, h->stream);  // kNoCertificate
            ++h->launches;
            if ((st = certify_tiles(h, base, tiles, T, maxA, maxB, tk_cache, want, target_bits, d_q, d_sc)))
                return st;
            if ((st = read_back(h, {{s_ce.data(), d_sc, tile_bytes}}))) return st;
        }
    }
    mark(h, kScale);  // statistics, certificate, features and the MLP count with the scale stage
    if (mode < 0) {  // features only
        if (feat_out)
            launch_sm_copy(d_feat, feat_out, ntiles * kFeatures * 4, h->stream);
        if (sa_out) launch_sm_copy(d_sa, sa_out, ntiles * 4, h->stream);
        if (ntiles_out) *ntiles_out = ntiles;
        return OZ2_OK;
    }

    // ---- per-tile s
    if (use_mlp) {
        // the MLP's s of a tile is the largest over the tile and its neighbours in the same
        // problem: one tile's statistics are noisy, its neighbours' see most of the same rows
        // and columns
        std::vector<int> pooled(ntiles);
        int64_t t0 = 0;
        for (size_t q = 0; q < base.size(); ++q) {
            const int64_t na = ceil_div(base[q].m, T), nbp = ceil_div(base[q].n, T);
            for (int64_t J = 0; J < nbp; ++J)
                for (int64_t I = 0; I < na; ++I) {
                    int v = 0;
                    for (int64_t dJ = -1; dJ <= 1; ++dJ)
                        for (int64_t dI = -1; dI <= 1; ++dI) {
                            const int64_t I2 = I + dI, J2 = J + dJ;
                            if (I2 >= 0 && I2 < na && J2 >= 0 && J2 < nbp) v = std::max(v, s_ml[t0 + J2 * na + I2]);
                        }
                    pooled[t0 + J * na + I] = v;
                }
            t0 += na * nbp;
        }
        s_ml.swap(pooled);
    }
    // the arbiter: the smaller of the analytic and the certified s (both meet the target)
    std::vector<int> s_jd(ntiles);
    for (int64_t t = 0; t < ntiles; ++t) s_jd[t] = certify ? std::min(s_an[t], std::max(s_ce[t], 2)) : s_an[t];
    std::vector<int> s_tile(ntiles);
    std::vector<int> prob_max(base.size(), 2);
    for (int64_t t = 0; t < ntiles; ++t) prob_max[tiles[t].prob] = std::max(prob_max[tiles[t].prob], s_jd[t]);
    for (int64_t t = 0; t < ntiles; ++t) {
        const int q = tiles[t].prob;
        int sv;
        switch (mode) {
            // the probe and the rerun need C's old values gone (beta = 0): other problems keep
            // the arbiter's s
            // a tile with a certificate takes it (rigorous, within about a modulus of the smallest
            // s that meets the target); the MLP chooses for the others, below the analytic s
            case 0:
                sv = use_mlp && base[q].beta[0] == 0.0 && s_ce[t] == kNoCertificate ? std::min(s_ml[t], s_jd[t])
                                                                                     : s_jd[t];
                break;
            case 1:
            case 4: sv = s_jd[t]; break;
            case 2:
            case 5: sv = prob_max[q]; break;
            default: sv = fixed_s[q]; break;
        }
        if (sv >= kNativeS) {
            s_tile[t] = kNativeS;
            continue;
        }
        // never below the smallest s that k admits
        const std::vector<int>& tk = tk_cache[base[q].k];
        while (sv < kMaxModuliExt && tk[sv] == 0) ++sv;
        s_tile[t] = std::max(2, std::min(kMaxModuliExt, sv));
    }
    if (mode == 0 || mode == 4) {
        // Per problem, the cheaper of its tiles as chosen and one whole-problem task (a larger s
        // only adds bits; native FP64 always meets the target). Work per tile ~ s mb nb k for an
        // emulated tile (a tile task costing kTileTax more than the same work in a whole-problem
        // task: more splits of the same panels, shorter GEMM tasks) and ~ kNativeCost mb nb k
        // for a native one (per-tile cuBLAS calls kTileTax more than one whole call). Measured
        // on B200: native FP64 costs as much as about 63 moduli of emulation.
        constexpr double kTileTax = 1.12, kNativeCost = 63.0;
        std::vector<double> tiles_cost(base.size(), 0.0), area(base.size(), 0.0);
        std::vector<int> hi(base.size(), 0);
        for (int64_t t = 0; t < ntiles; ++t) {
            const int q = tiles[t].prob;
            const double a = static_cast<double>(tiles[t].mb) * tiles[t].nb;
            const int sv = s_tile[t];
            tiles_cost[q] += kTileTax * a * (sv >= kNativeS ? kNativeCost : sv);
            area[q] += a;
            hi[q] = std::max(hi[q], sv);
        }
        std::vector<int> whole(base.size(), 0);  // 0 keep the tiles, else the s of one task
        for (size_t q = 0; q < base.size(); ++q) {
            const double emu = hi[q] <= kMaxModuliExt ? hi[q] * area[q] : 1e300;
            const double nat = kNativeCost * area[q];
            if (std::min(emu, nat) <= tiles_cost[q]) whole[q] = emu <= nat ? hi[q] : kNativeS;
        }
        for (int64_t t = 0; t < ntiles; ++t)
            if (whole[tiles[t].prob]) s_tile[t] = whole[tiles[t].prob];
    }

    // ---- phase 2: tiles with their s, panels split once per (panel, s); batches by budget
    std::vector<int64_t> prob_tiles(base.size(), 0), native_count(base.size(), 0);
    for (const TileRef& r : tiles) ++prob_tiles[r.prob];
    auto run_tiles = [&](const std::vector<int64_t>& which_all, const std::vector<int>& svals_all) -> int {
        // tiles that no moduli set brings to the target: native FP64 GEMM, one call per problem
        // when all its tiles go this way
        std::vector<int64_t> which, native;
        std::vector<int> svals;
        for (size_t i = 0; i < which_all.size(); ++i) {
            if (svals_all[i] >= kNativeS) {
                native.push_back(which_all[i]);
            } else {
                which.push_back(which_all[i]);
                svals.push_back(svals_all[i]);
            }
        }
        if (!native.empty()) {
            // no emulated tile shares data with them: they run beside the rest of the call
            int stf = native_fork(h);
            if (stf) return stf;
            h->nat_pending = true;
            if (h->profiling) OZ2_CUDA(h, cudaEventRecord(h->nat_t0, h->nat_stream));
            std::fill(native_count.begin(), native_count.end(), 0);
            for (int64_t t : native) ++native_count[tiles[t].prob];
            std::vector<bool> whole_done(base.size(), false);
            // other native tiles by (problem, row of tiles), in column order
            std::map<std::pair<int, int64_t>, std::vector<int64_t>> rows_of;
            for (int64_t t : native) {
                const TileRef& r = tiles[t];
                const Prob& p = base[r.prob];
                h->astats[8] += 1;
                h->astats[9] += r.mb * r.nb * p.k;
                if (native_count[r.prob] == prob_tiles[r.prob]) {
                    if (whole_done[r.prob]) continue;
                    whole_done[r.prob] = true;
                    const int st2 = native_gemm(h, h->nat_stream, p, 0, 0, p.m, p.n);
                    if (st2) return st2;
                } else {
                    rows_of[{r.prob, r.i0}].push_back(t);
                }
            }
            for (auto& kv : rows_of) {
                std::vector<int64_t>& ts = kv.second;
                std::sort(ts.begin(), ts.end(), [&](int64_t x, int64_t y) { return tiles[x].j0 < tiles[y].j0; });
                const Prob& p = base[kv.first.first];
                size_t a = 0;
                while (a < ts.size()) {
                    // a run of adjacent full-width tiles goes in one batched call
                    size_t b = a + 1;
                    while (b < ts.size() && tiles[ts[b]].j0 == tiles[ts[b - 1]].j0 + T && tiles[ts[b]].nb == T &&
                           tiles[ts[a]].nb == T)
                        ++b;
                    const TileRef& r = tiles[ts[a]];
                    const int st2 = b - a > 1 ? native_gemm_row(h, h->nat_stream, p, r.i0, r.j0, r.mb, T,
                                                                static_cast<int64_t>(b - a))
                                              : native_gemm(h, h->nat_stream, p, r.i0, r.j0, r.mb, r.nb);
                    if (st2) return st2;
                    a = b;
                }
            }
            if (h->profiling) {
                OZ2_CUDA(h, cudaEventRecord(h->nat_t1, h->nat_stream));
                OZ2_CUDA(h, cudaEventSynchronize(h->nat_t1));
                float ms = 0.0f;
                OZ2_CUDA(h, cudaEventElapsedTime(&ms, h->nat_t0, h->nat_t1));
                h->native_ms += ms;
            }
        }
        std::vector<std::unique_ptr<Prob>> probs;  // one per (problem, s)
        std::map<std::pair<int, int>, Prob*> prob_for;
        auto get_prob = [&](int q, int sv) -> Prob* {
            auto key = std::make_pair(q, sv);
            auto it = prob_for.find(key);
            if (it != prob_for.end()) return it->second;
            auto np = std::make_unique<Prob>(base[q]);
            const Plan* plan;
            if (get_plan(h, sv, base[q].k, &plan, true)) return nullptr;
            np->plan = plan;
            Prob* raw = np.get();
            probs.push_back(std::move(np));
            prob_for[key] = raw;
            return raw;
        };
        // the first workspace holds phase-1 data; the second may use what is left
        size_t limit = h->ws_limit;
        if (!limit) {
            size_t free_b = 0, total = 0;
            if (cudaMemGetInfo(&free_b, &total) != cudaSuccess) return fail(h, OZ2_ECUDA, "oz2: cudaMemGetInfo");
            free_b += h->ws2_size;
            const size_t reserve = (size_t{512} << 20) + total / 32;
            limit = free_b > reserve ? free_b - reserve : 0;
            // a batch of 16 GiB of planes and residues keeps every SM busy for milliseconds; more
            // only takes memory from the rest of the process (the caller's tensors, other calls)
            limit = std::min(limit, size_t{16} << 30);
        }
        // a problem whose tiles all run here at one s is one task: its GEMM jobs then share the
        // planes through the L2 across the whole problem, as in a plain call
        struct Unit {
            int64_t tile;  // -1: the whole problem
            int prob, s;
        };
        std::vector<Unit> units;
        {
            std::vector<int> common(base.size(), 0);  // 0 unseen, -1 mixed, else the s
            std::vector<int64_t> seen(base.size(), 0);
            for (size_t u = 0; u < which.size(); ++u) {
                const int q = tiles[which[u]].prob;
                common[q] = seen[q] == 0 ? svals[u] : (common[q] == svals[u] ? common[q] : -1);
                ++seen[q];
            }
            std::vector<bool> emitted(base.size(), false);
            for (size_t u = 0; u < which.size(); ++u) {
                const int q = tiles[which[u]].prob;
                bool whole = prob_tiles[q] > 1 && seen[q] == prob_tiles[q] && common[q] > 0;
                if (whole) {  // and only while the whole problem fits well inside the budget
                    const Prob& p = base[q];
                    const size_t bytes = static_cast<size_t>(common[q]) *
                                         (plane_geom(p.m, p.k, kGemmIPad).plane_bytes +
                                          plane_geom(p.n, p.k, kGemmJ).plane_bytes + p.n * round_up(p.m, 32));
                    whole = bytes <= limit / 2;
                }
                if (!whole) {
                    units.push_back(Unit{which[u], q, svals[u]});
                } else if (!emitted[q]) {
                    emitted[q] = true;
                    units.push_back(Unit{-1, q, common[q]});
                }
            }
        }
        size_t i = 0;
        while (i < units.size()) {
            // one batch: units until the budget is reached
            std::map<std::tuple<int, int, int>, std::pair<size_t, bool>> panels;  // (panel, side, s) -> offset
            size_t off2 = 0;
            auto carve2 = [&](size_t bytes) {
                const size_t o = off2;
                off2 += align256(bytes);
                return o;
            };
            struct Slot {
                size_t a, b, r;  // offsets of the A planes, B planes and residues
            };
            std::vector<Slot> batch;
            size_t start = i;
            for (; i < units.size(); ++i) {
                const Unit& un = units[i];
                const int sv = un.s;
                const Prob& p = base[un.prob];
                const int64_t mb = un.tile < 0 ? p.m : tiles[un.tile].mb, nb = un.tile < 0 ? p.n : tiles[un.tile].nb;
                const size_t pa = static_cast<size_t>(sv) * plane_geom(mb, p.k, kGemmIPad).plane_bytes;
                const size_t pb = static_cast<size_t>(sv) * plane_geom(nb, p.k, kGemmJ).plane_bytes;
                const size_t rs = static_cast<size_t>(sv) * nb * round_up(mb, 32);
                const size_t items = 2 * sizeof(SplitItem) + sizeof(GemmItem) + sizeof(CrtItem) + 2048;
                if (un.tile < 0) {
                    const size_t add = align256(pa) + align256(pb) + align256(rs) + items;
                    if (i > start && off2 + add + (1 << 20) > limit) break;
                    const size_t oa = carve2(pa), ob = carve2(pb);
                    batch.push_back(Slot{oa, ob, carve2(rs)});
                    h->gbytes[0] += static_cast<int64_t>(pa + pb);
                    h->gbytes[1] += static_cast<int64_t>(rs);
                    continue;
                }
                const TileRef& r = tiles[un.tile];
                const bool newa = !panels.count({r.ia, 0, sv}), newb = !panels.count({r.jb, 1, sv});
                const size_t add = (newa ? align256(pa) : 0) + (newb ? align256(pb) : 0) + align256(rs) + items;
                if (i > start && off2 + add + (1 << 20) > limit) break;
                if (newa) panels[{r.ia, 0, sv}] = {carve2(pa), true};
                if (newb) panels[{r.jb, 1, sv}] = {carve2(pb), true};
                h->gbytes[0] += static_cast<int64_t>((newa ? pa : 0) + (newb ? pb : 0));
                h->gbytes[1] += static_cast<int64_t>(rs);
                batch.push_back(Slot{panels[{r.ia, 0, sv}].first, panels[{r.jb, 1, sv}].first, carve2(rs)});
            }
            const size_t obase_desc = off2;
            h->gbytes[2] += 1;
            const size_t need = off2 + align256(batch.size() * (2 * sizeof(SplitItem) + sizeof(GemmItem) +
                                                                sizeof(CrtItem) + 1024) + 8192);
            int st2 = ensure_ws2(h, need);
            if (st2) return st2;
            std::vector<Task> tasks;
            std::map<std::tuple<int, int, int>, bool> split_done;
            for (size_t b = 0; b < batch.size(); ++b) {
                const Unit& un = units[start + b];
                const int sv = un.s;
                Prob* p = get_prob(un.prob, sv);
                if (!p) return fail(h, OZ2_EINTERNAL, "oz2: no plan for adaptive tile");
                Task tk{};
                tk.p = p;
                if (un.tile < 0) {
                    tk.i0 = tk.j0 = 0;
                    tk.mb = p->m;
                    tk.nb = p->n;
                    tk.split_a = tk.split_b = true;
                    h->astats[1] += static_cast<int64_t>(sv) * prob_tiles[un.prob];
                } else {
                    const TileRef& r = tiles[un.tile];
                    tk.i0 = r.i0;
                    tk.j0 = r.j0;
                    tk.mb = r.mb;
                    tk.nb = r.nb;
                    tk.split_a = !split_done[{r.ia, 0, sv}];
                    tk.split_b = !split_done[{r.jb, 1, sv}];
                    split_done[{r.ia, 0, sv}] = true;
                    split_done[{r.jb, 1, sv}] = true;
                    h->astats[1] += sv;
                }
                tk.maxA = maxA(un.prob);
                tk.maxB = maxB(un.prob);
                tk.planesA = reinterpret_cast<int8_t*>(h->ws2 + batch[b].a);
                tk.planesB = reinterpret_cast<int8_t*>(h->ws2 + batch[b].b);
                tk.resid = h->ws2 + batch[b].r;
                tk.ldr = round_up(tk.mb, 32);
                tasks.push_back(tk);
                h->astats[7] += static_cast<int64_t>(sv) * tk.mb * tk.nb * base[un.prob].k;
            }
            std::vector<const Prob*> bp;
            for (auto& up : probs) bp.push_back(up.get());
            const GemmConfig cfg = config_for(h, bp);
            h->last_cfg = cfg;
            Program prog;
            plan_tasks(prog, tasks, cfg);
            if (obase_desc + prog.blob.size() > h->ws2_size)
                return fail(h, OZ2_EINTERNAL, "oz2: descriptor region too small");
            if ((st2 = check_grid(h, prog))) return st2;
            if ((st2 = upload(h, prog, h->ws2 + obase_desc))) return st2;
            mark(h, kBegin);
            issue(h, prog, h->ws2 + obase_desc);
        }
        return OZ2_OK;
    };
    std::vector<int64_t> all(ntiles);
    for (int64_t t = 0; t < ntiles; ++t) all[t] = t;
    h->astats[0] = ntiles;
    if ((st = run_tiles(all, s_tile))) return st;

    // ---- probe (MLP mode, problems with beta = 0) and rerun at the analytic s
    if (mode == 0) {
        std::vector<ProbeItem> pi;
        int64_t blocks = 0;
        // the longest tiles (largest k) first, so that the short ones fill the last wave; within
        // a problem, tiles of one row panel next to each other share its rows of A in the L2
        std::vector<int64_t> porder(ntiles);
        for (int64_t t = 0; t < ntiles; ++t) porder[t] = t;
        std::stable_sort(porder.begin(), porder.end(), [&](int64_t x, int64_t y) {
            const int64_t kx = base[tiles[x].prob].k, ky = base[tiles[y].prob].k;
            if (kx != ky) return kx > ky;
            return std::make_pair(tiles[x].prob, tiles[x].i0) < std::make_pair(tiles[y].prob, tiles[y].i0);
        });
        for (const int64_t t : porder) {
            const TileRef& r = tiles[t];
            const Prob& p = base[r.prob];
            if (h->probe_kind == 3) break;  // no probe: the MLP's s stands (for measurements)
            if (p.beta[0] != 0.0 || s_tile[t] >= s_jd[t]) continue;  // the arbiter's s needs no probe
            ProbeItem it{};
            it.a_rowc = is_n(p.ta);
            it.b_rowc = !is_n(p.tb);
            it.A = p.A + (it.a_rowc ? r.i0 : r.i0 * p.lda);
            it.B = p.B + (it.b_rowc ? r.j0 : r.j0 * p.ldb);
            it.C = p.C + r.i0 + r.j0 * p.ldc;
            it.lda = p.lda;
            it.ldb = p.ldb;
            it.ldc = p.ldc;
            it.mt = r.mb;
            it.nt = r.nb;
            it.k = p.k;
            it.alpha = p.alpha[0];
            it.tol_scale = static_cast<double>(p.k) * std::ldexp(1.0, -target_bits);
            it.seed = 0x5DEECE66Dull * static_cast<uint64_t>(t + 1) + static_cast<uint64_t>(r.prob);
            it.tile = static_cast<int>(t);
            blocks += probe_item_blocks(it, blocks);
            pi.push_back(it);
        }
        if (!pi.empty()) {
            unsigned char* pd = ws + odesc;  // phase-1 descriptors are consumed by now (stream order)
            // Freivalds items: the same tiles, their column maxima and 3 kFreivaldsVecs k doubles
            // of work each in the tile workspace, whose planes and residues are dead by now
            std::vector<FreivaldsItem> f1, f2;
            int64_t fb1 = 0, fb2 = 0;
            if (h->probe_kind != 0) {
                size_t fwork = 0;
                for (const ProbeItem& q : pi) fwork += align256(3 * kFreivaldsVecs * q.k * sizeof(double));
                if ((st = ensure_ws2(h, fwork))) return st;
                size_t fo = 0;
                for (const ProbeItem& q : pi) {
                    const TileRef& r = tiles[q.tile];
                    FreivaldsItem it{};
                    it.A = q.A;
                    it.B = q.B;
                    it.C = q.C;
                    it.maxb = maxB(r.prob) + r.j0;
                    it.work = reinterpret_cast<double*>(h->ws2 + fo);
                    fo += align256(3 * kFreivaldsVecs * q.k * sizeof(double));
                    it.lda = q.lda;
                    it.ldb = q.ldb;
                    it.ldc = q.ldc;
                    it.mt = q.mt;
                    it.nt = q.nt;
                    it.k = q.k;
                    it.a_rowc = q.a_rowc;
                    it.b_rowc = q.b_rowc;
                    it.alpha = q.alpha;
                    it.tol_scale = q.tol_scale;
                    it.seed = q.seed;
                    it.tile = q.tile;
                    f1.push_back(it);
                    fb1 += freivalds_blocks_pass1(f1.back(), fb1);
                    f2.push_back(it);
                    fb2 += freivalds_blocks_pass2(f2.back(), fb2);
                }
            }
            const size_t o1 = align256(pi.size() * sizeof(ProbeItem));
            const size_t o2 = o1 + align256(f1.size() * sizeof(FreivaldsItem));
            if (h->probe_kind != 1 && (st = put_blob(h, pi.data(), pi.size() * sizeof(ProbeItem), pd))) return st;
            if (h->probe_kind != 0) {
                if ((st = put_blob(h, f1.data(), f1.size() * sizeof(FreivaldsItem), pd + o1))) return st;
                if ((st = put_blob(h, f2.data(), f2.size() * sizeof(FreivaldsItem), pd + o2))) return st;
            }
            mark(h, kBegin);
            if (h->probe_kind != 1) {
                launch_probe(reinterpret_cast<const ProbeItem*>(pd), static_cast<int>(pi.size()), blocks, d_fail,
                             h->stream);
                ++h->launches;
            }
            if (h->probe_kind != 0) {
                launch_freivalds(reinterpret_cast<const FreivaldsItem*>(pd + o1), fb1,
                                 reinterpret_cast<const FreivaldsItem*>(pd + o2), fb2, static_cast<int>(f1.size()),
                                 d_fail, h->stream);
                h->launches += 2;
            }
            mark(h, kProbe);
            std::vector<int> failed(ntiles);
            if ((st = read_back(h, {{failed.data(), d_fail, static_cast<size_t>(ntiles) * 4}}))) return st;
            h->astats[2] = static_cast<int64_t>(pi.size());
            std::vector<int64_t> redo;
            std::vector<int> redo_s;
            for (int64_t t = 0; t < ntiles; ++t)
                if (failed[t]) {
                    redo.push_back(t);
                    redo_s.push_back(s_jd[t]);
                }
            h->astats[3] = static_cast<int64_t>(redo.size());
            if (!redo.empty()) {
                // beta = 0 for every probed tile, so recomputing C overwrites the failed values
                int64_t extra = 0;
                for (size_t q = 0; q < redo.size(); ++q) extra += redo_s[q];
                h->astats[4] = extra;
                if ((st = run_tiles(redo, redo_s))) return st;
            }
        }
    }
    for (int64_t t = 0; t < ntiles; ++t) h->astats[5] += s_jd[t];
    h->astats[6] = use_mlp ? 1 : 0;
    return OZ2_OK;
}

int validate_grouped(oz2_handle h, int count, const oz2_dgemm_problem* pr, std::vector<Prob>& out) {
    out.clear();
    out.reserve(count);
    for (int i = 0; i < count; ++i) {
        const oz2_dgemm_problem& q = pr[i];
        int st = check_args(h, q.ta, q.tb, q.m, q.n, q.k, q.lda, q.ldb, q.ldc);
        if (st) return fail(h, st, "oz2: problem " + std::to_string(i) + ": " + h->err);
    }
    for (int i = 0; i < count; ++i) {
        const oz2_dgemm_problem& q = pr[i];
        if (q.m == 0 || q.n == 0 || q.k == 0 || q.alpha == 0.0) continue;
        const Plan* plan;
        int st = get_plan(h, q.num_moduli, q.k, &plan);
        if (st) return fail(h, st, "oz2: problem " + std::to_string(i) + ": " + h->err);
        out.push_back(Prob{q.ta, q.tb, q.m, q.n, q.k, {q.alpha, 0.0}, {q.beta, 0.0}, q.A, q.lda, q.B, q.ldb, q.C, q.ldc, 1,
                           plan});
    }
    return OZ2_OK;
}


int validate_adaptive(oz2_handle h, int count, const oz2_dgemm_problem* pr, std::vector<Prob>& out,
                      std::vector<int>& fixed_s, bool need_fixed) {
    out.clear();
    fixed_s.clear();
    for (int i = 0; i < count; ++i) {
        const oz2_dgemm_problem& q = pr[i];
        int st = check_args(h, q.ta, q.tb, q.m, q.n, q.k, q.lda, q.ldb, q.ldc);
        if (st) return fail(h, st, "oz2: problem " + std::to_string(i) + ": " + h->err);
    }
    for (int i = 0; i < count; ++i) {
        const oz2_dgemm_problem& q = pr[i];
        if (q.m == 0 || q.n == 0 || q.k == 0 || q.alpha == 0.0) continue;
        if (need_fixed) {  // mode 3 takes the extended sets too (s up to 32)
            const Plan* plan;
            int st = get_plan(h, q.num_moduli, q.k, &plan, true);
            if (st) return fail(h, st, "oz2: problem " + std::to_string(i) + ": " + h->err);
        }
        out.push_back(Prob{q.ta, q.tb, q.m, q.n, q.k, {q.alpha, 0.0}, {q.beta, 0.0}, q.A, q.lda, q.B, q.ldb, q.C, q.ldc, 1,
                           nullptr});
        fixed_s.push_back(q.num_moduli);
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
    if (e == cudaSuccess) e = cudaMalloc(&h->d_err, 4 * sizeof(int));  // error word + scratch words
    if (e == cudaSuccess) e = cudaMemset(h->d_err, 0, 4 * sizeof(int));
    if (e == cudaSuccess) e = prepare_gemm_kernels();
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
    drop_graphs(h);
    if (h->ws) cudaFree(h->ws);
    if (h->d_err) cudaFree(h->d_err);
    for (cudaEvent_t e : h->pool) cudaEventDestroy(e);
    for (int i = 0; i < kRing; ++i) {
        if (h->ring_host[i]) cudaFreeHost(h->ring_host[i]);
        if (h->ring_ev[i]) cudaEventDestroy(h->ring_ev[i]);
    }
    if (h->rb_host) cudaFreeHost(h->rb_host);
    if (h->cap_stream) cudaStreamDestroy(h->cap_stream);
    if (h->d_mlp) cudaFree(h->d_mlp);
    if (h->ws2) cudaFree(h->ws2);
    if (h->cublas) cublasDestroy(h->cublas);
    if (h->nat_stream) cudaStreamDestroy(h->nat_stream);
    if (h->xfer) cudaStreamDestroy(h->xfer);
    if (h->xfer_in) cudaEventDestroy(h->xfer_in);
    for (cudaEvent_t e : {h->nat_fork, h->nat_join, h->nat_t0, h->nat_t1})
        if (e) cudaEventDestroy(e);
    delete h;
    return OZ2_OK;
}

int oz2_set_stream(oz2_handle h, void* stream) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    h->stream = static_cast<cudaStream_t>(stream);
    drop_graphs(h);
    return OZ2_OK;
}

// ref src/ozaki2_gpu.hpp:739-760
int oz2_dgemm(oz2_handle h, char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A,
              int64_t lda, const double* B, int64_t ldb, double beta, double* C, int64_t ldc, int num_moduli,
              void* const* deps, int ndeps, void* done) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    h->marks.clear();
    if (h->plans.size() > 8192) h->plans.clear();  // between calls only: plans are borrowed during one
    int st = check_args(h, ta, tb, m, n, k, lda, ldb, ldc);
    if (st) return st;
    if ((st = begin_call(h, deps, ndeps))) return st;
    if (m == 0 || n == 0) return end_call(h, done);
    const double be[2] = {beta, 0.0};
    if (k == 0 || alpha == 0.0) {
        launch_scale_c(C, ldc, m, n, be, false, h->stream);
        ++h->launches;
        return end_call(h, done);
    }
    const Plan* plan;
    if ((st = get_plan(h, num_moduli, k, &plan))) return st;
    const Prob p{ta, tb, m, n, k, {alpha, 0.0}, {beta, 0.0}, A, lda, B, ldb, C, ldc, 1, plan};
    if ((st = run_single(h, p))) return st;
    return end_call(h, done);
}

// The reference's Ozaki Scheme I comparison baseline, oz1::Ozaki1::gemm
// (benchmarks/ozaki1_gpu.hpp:85-147): C = A B, A and B column-major and not transposed.
int oz2_ozaki1_dgemm(oz2_handle h, int64_t m, int64_t n, int64_t k, const double* A, int64_t lda, const double* B,
                     int64_t ldb, double* C, int64_t ldc, int L) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    h->marks.clear();
    if (L < 2 || L > 9) return fail(h, OZ2_EINVAL, "oz2: L must be in [2, 9]");
    int st = check_args(h, 'N', 'N', m, n, k, lda, ldb, ldc);
    if (st) return st;
    if (k * 4096 >= (int64_t{1} << 31)) return fail(h, OZ2_EINVAL, "oz2: k too large for the int32 digit products");
    if ((st = begin_call(h, nullptr, 0))) return st;
    if (m == 0 || n == 0) return end_call(h, nullptr);
    if (k == 0) {  // C = A B = 0
        const double zero[2] = {0.0, 0.0};
        launch_scale_c(C, ldc, m, n, zero, false, h->stream);
        ++h->launches;
        return end_call(h, nullptr);
    }
    const int tk = 7 * L - 2, npairs = L * (L + 1) / 2;
    const PlaneGeom ga = plane_geom(m, k, kGemmIPad), gb = plane_geom(n, k, kGemmJ);
    size_t off = 0;
    auto carve = [&](size_t bytes) {
        const size_t o = off;
        off += align256(bytes);
        return o;
    };
    const size_t o_ma = carve(static_cast<size_t>(m) * 8), o_mb = carve(static_cast<size_t>(n) * 8);
    const size_t o_acc = carve(static_cast<size_t>(L) * m * n * 8);
    const size_t zero_end = off;
    const size_t o_pa = carve(static_cast<size_t>(L) * ga.plane_bytes), o_pb = carve(static_cast<size_t>(L) * gb.plane_bytes);
    const size_t o_desc = carve(64 << 10);
    if ((st = ensure_workspace(h, off))) return st;
    auto* maxA = reinterpret_cast<unsigned long long*>(h->ws + o_ma);
    auto* maxB = reinterpret_cast<unsigned long long*>(h->ws + o_mb);
    auto* acc = reinterpret_cast<int64_t*>(h->ws + o_acc);
    auto* planesA = reinterpret_cast<int8_t*>(h->ws + o_pa);
    auto* planesB = reinterpret_cast<int8_t*>(h->ws + o_pb);

    const Prob p{'N', 'N', m, n, k, {1.0, 0.0}, {0.0, 0.0}, A, lda, B, ldb, C, ldc, 1, nullptr};
    Program prog;
    Op ms;
    ms.kind = Op::Memset;
    ms.ptr = h->ws;
    ms.bytes = zero_end;
    prog.ops.push_back(ms);
    std::vector<ScaleItem> sc{scale_item(p, true, maxA), scale_item(p, false, maxB)};
    plan_scale(h, prog, sc);
    for (int side = 0; side < 2; ++side) {  // digits: A rows contiguous, B columns k-contiguous
        SplitItem it{};
        it.X = side ? B : A;
        it.ldx = side ? ldb : lda;
        it.rows = side ? n : m;
        it.k = k;
        it.row_contig = side ? 0 : 1;
        it.tk = tk;
        it.s = L;
        it.maxbits = side ? maxB : maxA;
        it.planes = side ? planesB : planesA;
        const PlaneGeom& g = side ? gb : ga;
        it.rows_pad = g.rows_pad;
        it.kb_total = g.kb_total;
        it.plane_bytes = g.plane_bytes;
        Op op;
        op.kind = Op::Slice;
        op.count = 1;
        op.blocks = split_item_blocks(it, 0);
        op.off = prog.add(&it, sizeof it);
        prog.ops.push_back(op);
    }
    GemmConfig cfg;  // BN 256, raster 16
    GemmItem g{};
    g.planes_i = planesA;
    g.planes_j = planesB;
    g.pstride_i = ga.plane_bytes;
    g.pstride_j = gb.plane_bytes;
    g.m = m;
    g.n = n;
    g.kb_total = ga.kb_total;
    g.tiles_i = static_cast<int>(gemm_tiles_i(m, cfg.bn));
    g.tiles_j = static_cast<int>(ceil_div(n, kGemmJ));
    g.tiles = static_cast<int64_t>(g.tiles_i) * g.tiles_j;
    g.s = npairs;
    g.groups = 1;
    g.job0 = 0;
    g.acc = acc;
    g.acc_ld = n;
    g.acc_plane = m * n;
    for (int d = 0, t = 0; d < L; ++d)
        for (int a = 0; a <= d; ++a, ++t) {
            g.pair_a[t] = static_cast<uint8_t>(a);
            g.pair_b[t] = static_cast<uint8_t>(d - a);
            g.pair_d[t] = static_cast<uint8_t>(d);
        }
    Op go;
    go.kind = Op::GemmOz1;
    go.count = 1;
    go.jobs = g.tiles * npairs;
    go.cfg = cfg;
    go.off = prog.add(&g, sizeof g);
    prog.ops.push_back(go);
    if ((st = check_grid(h, prog))) return st;
    unsigned char* dev_desc = h->ws + o_desc;
    if (prog.blob.size() > (64u << 10)) return fail(h, OZ2_EINTERNAL, "oz2: descriptor region too small");
    if ((st = upload(h, prog, dev_desc))) return st;
    issue(h, prog, dev_desc);
    launch_oz1_horner(acc, m, n, L, maxA, maxB, tk, C, ldc, h->stream);
    ++h->launches;
    return end_call(h, nullptr);
}

// ref src/ozaki2_gpu.hpp:764-786 (plan for 2k: the 3M sums double the inner products)
int oz2_zgemm(oz2_handle h, char ta, char tb, int64_t m, int64_t n, int64_t k, const double* alpha,
              const double* A, int64_t lda, const double* B, int64_t ldb, const double* beta, double* C,
              int64_t ldc, int num_moduli, void* const* deps, int ndeps, void* done) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    if (!alpha || !beta) return fail(h, OZ2_EINVAL, "oz2: null alpha or beta");
    h->marks.clear();
    if (h->plans.size() > 8192) h->plans.clear();
    int st = check_args(h, ta, tb, m, n, k, lda, ldb, ldc);
    if (st) return st;
    if ((st = begin_call(h, deps, ndeps))) return st;
    if (m == 0 || n == 0) return end_call(h, done);
    if (k == 0 || (alpha[0] == 0.0 && alpha[1] == 0.0)) {
        launch_scale_c(C, ldc, m, n, beta, true, h->stream);
        ++h->launches;
        return end_call(h, done);
    }
    if (k > std::numeric_limits<int64_t>::max() / 2) return fail(h, OZ2_EINVAL, "oz2: k too large");
    const Plan* plan;
    if ((st = get_plan(h, num_moduli, 2 * k, &plan))) return st;
    const Prob p{ta, tb, m, n, k, {alpha[0], alpha[1]}, {beta[0], beta[1]}, A, lda, B, ldb, C, ldc, 3, plan};
    if ((st = run_single(h, p))) return st;
    return end_call(h, done);
}

int oz2_dgemm_grouped(oz2_handle h, int count, const oz2_dgemm_problem* problems, void* const* deps, int ndeps,
                      void* done) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    if (count < 0 || (count > 0 && !problems)) return fail(h, OZ2_EINVAL, "oz2: bad problem list");
    h->marks.clear();
    if (h->plans.size() > 8192) h->plans.clear();
    // num_moduli = -1: the adaptive path (mode 0, DGEMM-level target) for those problems
    std::vector<oz2_dgemm_problem> fixed_list, adaptive_list;
    for (int i = 0; i < count; ++i) (problems[i].num_moduli == OZ2_S_ADAPTIVE ? adaptive_list : fixed_list).push_back(problems[i]);
    if (!adaptive_list.empty()) {
        if (h->graph_mode)
            return fail(h, OZ2_EINVAL, "oz2: num_moduli = -1 (adaptive) does not run in graph mode: the adaptive "
                                       "choice reads tile statistics back to the host");
        std::vector<Prob> fprobs, aprobs;
        std::vector<int> afixed;
        int st = validate_grouped(h, static_cast<int>(fixed_list.size()), fixed_list.data(), fprobs);
        if (st) return st;
        if ((st = validate_adaptive(h, static_cast<int>(adaptive_list.size()), adaptive_list.data(), aprobs, afixed,
                                    false)))
            return st;
        if ((st = begin_call(h, deps, ndeps))) return st;
        for (int i = 0; i < count; ++i) {  // k == 0 or alpha == 0: C = beta C
            const oz2_dgemm_problem& q = problems[i];
            if (q.m > 0 && q.n > 0 && (q.k == 0 || q.alpha == 0.0)) {
                const double be[2] = {q.beta, 0.0};
                launch_scale_c(q.C, q.ldc, q.m, q.n, be, false, h->stream);
                ++h->launches;
            }
        }
        if (!fprobs.empty() && (st = run_grouped(h, fprobs))) return st;
        if (!aprobs.empty()) {
            for (int q = 0; q < kAdaptiveStats; ++q) h->astats[q] = 0;
            for (int64_t& g : h->gbytes) g = 0;
            h->native_ms = 0.0;
            st = run_adaptive(h, aprobs, afixed, 53, 0);
            const int sj = native_join(h);
            if (st) return st;
            if (sj) return sj;
        }
        return end_call(h, done);
    }
    std::vector<Prob> probs;
    int st = validate_grouped(h, count, problems, probs);
    if (st) return st;
    if ((st = begin_call(h, deps, ndeps))) return st;
    for (int i = 0; i < count; ++i) {  // k == 0 or alpha == 0: C = beta C
        const oz2_dgemm_problem& q = problems[i];
        if (q.m > 0 && q.n > 0 && (q.k == 0 || q.alpha == 0.0)) {
            const double be[2] = {q.beta, 0.0};
            launch_scale_c(q.C, q.ldc, q.m, q.n, be, false, h->stream);
            ++h->launches;
        }
    }
    if (probs.empty()) return end_call(h, done);
    if (!h->graph_mode) {
        if ((st = run_grouped(h, probs))) return st;
        return end_call(h, done);
    }
    // graph mode: the same problem list (shapes, pointers, scalars) replays its graphs
    const unsigned char* raw = reinterpret_cast<const unsigned char*>(problems);
    const size_t raw_bytes = static_cast<size_t>(count) * sizeof(oz2_dgemm_problem);
    uint64_t key = 1469598103934665603ull;  // FNV-1a
    for (size_t i = 0; i < raw_bytes; ++i) key = (key ^ raw[i]) * 1099511628211ull;
    auto it = h->graphs.find(key);
    if (it != h->graphs.end() && it->second.problems.size() == raw_bytes &&
        std::memcmp(it->second.problems.data(), raw, raw_bytes) == 0) {
        mark(h, kBegin);
        for (auto e : it->second.execs) OZ2_CUDA(h, cudaGraphLaunch(e, h->stream));
        h->launches += it->second.kernels;
        mark(h, kCrt);
        return end_call(h, done);
    }
    if (h->graphs.size() >= 64) drop_graphs(h);
    GraphEntry fresh;
    fresh.problems.assign(raw, raw + raw_bytes);
    GraphEntry& ge = h->graphs[key];
    for (auto e : ge.execs) cudaGraphExecDestroy(e);
    for (auto b : ge.dev_blobs) cudaFree(b);
    ge = std::move(fresh);
    h->capturing = &ge;
    h->capture_ok = true;
    st = run_grouped(h, probs);
    const bool keep = h->capturing != nullptr && h->capture_ok;
    h->capturing = nullptr;
    if (st || !keep) drop_graphs(h);
    if (st) return st;
    return end_call(h, done);
}


int oz2_dgemm_adaptive(oz2_handle h, int count, const oz2_dgemm_problem* problems, int target_bits, int mode,
                       int64_t* stats) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    if (count < 0 || (count > 0 && !problems)) return fail(h, OZ2_EINVAL, "oz2: bad problem list");
    if (target_bits < 1 || target_bits > 120) return fail(h, OZ2_EINVAL, "oz2: target_bits must be in [1, 120]");
    if (mode < 0 || mode > 5) return fail(h, OZ2_EINVAL, "oz2: mode must be 0..5");
    h->marks.clear();
    if (h->plans.size() > 8192) h->plans.clear();
    std::vector<Prob> probs;
    std::vector<int> fixed_s;
    int st = validate_adaptive(h, count, problems, probs, fixed_s, mode == 3);
    if (st) return st;
    if ((st = begin_call(h, nullptr, 0))) return st;
    for (int i = 0; i < count; ++i) {
        const oz2_dgemm_problem& q = problems[i];
        if (q.m > 0 && q.n > 0 && (q.k == 0 || q.alpha == 0.0)) {
            const double be[2] = {q.beta, 0.0};
            launch_scale_c(q.C, q.ldc, q.m, q.n, be, false, h->stream);
            ++h->launches;
        }
    }
    for (int q = 0; q < kAdaptiveStats; ++q) h->astats[q] = 0;
    for (int64_t& g : h->gbytes) g = 0;
    h->native_ms = 0.0;
    if (!probs.empty()) st = run_adaptive(h, probs, fixed_s, target_bits, mode);
    const int sj = native_join(h);  // on every path: the stream must cover the native tiles
    if (st) return st;
    if (sj) return sj;
    if (stats)
        for (int q = 0; q < kAdaptiveStats; ++q) stats[q] = h->astats[q];
    return end_call(h, nullptr);
}

int oz2_tile_features(oz2_handle h, int count, const oz2_dgemm_problem* problems, int target_bits,
                      float* d_features, int* d_s_analytic, int64_t* ntiles) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    std::vector<Prob> probs;
    std::vector<int> fixed_s;
    int st = validate_adaptive(h, count, problems, probs, fixed_s, false);
    if (st) return st;
    int64_t nt = 0;
    if (!probs.empty() && (st = run_adaptive(h, probs, fixed_s, target_bits, -1, d_features, d_s_analytic, &nt)))
        return st;
    if (ntiles) *ntiles = nt;
    return end_call(h, nullptr);
}

int oz2_set_probe_kind(oz2_handle h, int kind) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    if (kind < 0 || kind > 3) return fail(h, OZ2_EINVAL, "oz2: probe kind must be 0, 1, 2 or 3");
    h->probe_kind = kind;
    return OZ2_OK;
}

int oz2_set_adaptive_options(oz2_handle h, int tile, float threshold) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    if (tile < 128 || tile % 128 || !(threshold > 0.0f && threshold <= 1.0f))
        return fail(h, OZ2_EINVAL, "oz2: tile must be a positive multiple of 128, threshold in (0, 1]");
    h->adaptive_tile = tile;
    h->mlp_threshold = threshold;
    return OZ2_OK;
}

int oz2_mlp_info(int* out4) {
    if (!out4) return fail(nullptr, OZ2_EINVAL, "oz2: null argument");
    out4[0] = kMlpParams;
    out4[1] = kFeatures;
    out4[2] = kClasses;
    out4[3] = kHidden;
    return OZ2_OK;
}

int oz2_mlp_set_weights(oz2_handle h, const float* params, int nparams) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    if (!params) {
        h->mlp_loaded = false;
        return OZ2_OK;
    }
    if (nparams != kMlpParams) return fail(h, OZ2_EINVAL, "oz2: wrong number of MLP parameters");
    if (!h->d_mlp) OZ2_CUDA(h, cudaMalloc(&h->d_mlp, kMlpParams * sizeof(float)));
    OZ2_CUDA(h, cudaMemcpyAsync(h->d_mlp, params, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    OZ2_CUDA(h, cudaStreamSynchronize(h->stream));
    h->mlp_loaded = true;
    return OZ2_OK;
}

int oz2_mlp_train(oz2_handle h, int count, const float* d_features, const int* d_labels, int epochs, float lr,
                  unsigned int seed, float* params, float* loss) {
    if (!h || !params || count <= 0 || epochs <= 0) return fail(h, OZ2_EINVAL, "oz2: bad training arguments");
    float* dp = nullptr;
    float* dl = nullptr;
    OZ2_CUDA(h, cudaMalloc(&dp, kMlpParams * sizeof(float)));
    cudaError_t e = cudaMalloc(&dl, static_cast<size_t>(epochs) * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpyAsync(dp, params, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        launch_mlp_train(dp, count, d_features, d_labels, epochs, lr, seed, dl, h->stream);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(params, dp, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess && loss)
        e = cudaMemcpyAsync(loss, dl, static_cast<size_t>(epochs) * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(dp);
    if (dl) cudaFree(dl);
    if (e != cudaSuccess) return cuda_fail(h, e, "oz2_mlp_train");
    return OZ2_OK;
}

int oz2_mlp_infer(oz2_handle h, const float* params, int count, const float* d_features, float threshold, int* d_s,
                  float* d_probs) {
    if (!h || !params || count < 0) return fail(h, OZ2_EINVAL, "oz2: bad inference arguments");
    float* dp = nullptr;
    OZ2_CUDA(h, cudaMalloc(&dp, kMlpParams * sizeof(float)));
    cudaError_t e = cudaMemcpyAsync(dp, params, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        launch_mlp_infer(dp, count, d_features, threshold, d_s, d_probs, h->stream);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(dp);
    if (e != cudaSuccess) return cuda_fail(h, e, "oz2_mlp_infer");
    return OZ2_OK;
}

int oz2_dd_reference(oz2_handle h, int64_t m, int64_t n, int64_t k, const double* A, int64_t lda, const double* B,
                     int64_t ldb, double* hi, double* lo, double* absab) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    if (m < 0 || n < 0 || k < 0 || lda < std::max<int64_t>(1, m) || ldb < std::max<int64_t>(1, k))
        return fail(h, OZ2_EINVAL, "oz2: bad dimensions");
    if (m == 0 || n == 0) return OZ2_OK;
    launch_dd_gemm_nn(m, n, k, A, lda, B, ldb, hi, lo, absab, h->stream);
    return end_call(h, nullptr);
}

int oz2_error_ratio(oz2_handle h, int64_t m, int64_t n, int64_t k, const double* C, int64_t ldc, const double* hi,
                    const double* lo, const double* absab, int target_bits, float* out) {
    if (!h || !out) return fail(h, OZ2_EINVAL, "oz2: null argument");
    if (m <= 0 || n <= 0 || ldc < m) return fail(h, OZ2_EINVAL, "oz2: bad dimensions");
    OZ2_CUDA(h, cudaMemsetAsync(h->d_err + 1, 0, sizeof(unsigned int), h->stream));
    launch_error_ratio(m, n, C, ldc, hi, lo, absab, static_cast<double>(k) * std::ldexp(1.0, -target_bits),
                       reinterpret_cast<unsigned int*>(h->d_err + 1), h->stream);
    unsigned int bits = 0;
    OZ2_CUDA(h, cudaMemcpyAsync(&bits, h->d_err + 1, sizeof bits, cudaMemcpyDeviceToHost, h->stream));
    OZ2_CUDA(h, cudaStreamSynchronize(h->stream));
    std::memcpy(out, &bits, sizeof bits);
    return OZ2_OK;
}

int oz2_accuracy(oz2_handle h, int64_t m, int64_t n, const double* C, int64_t ldc, const double* hi,
                 const double* lo, double* max_ulp, int64_t* correctly_rounded) {
    if (!h || !max_ulp || !correctly_rounded) return fail(h, OZ2_EINVAL, "oz2: null argument");
    if (m <= 0 || n <= 0 || ldc < m) return fail(h, OZ2_EINVAL, "oz2: bad dimensions");
    // d_err[2..3] hold the 64-bit count, d_err[1] the float bits of the maximum
    OZ2_CUDA(h, cudaMemsetAsync(h->d_err + 1, 0, 3 * sizeof(int), h->stream));
    auto* cnt = reinterpret_cast<unsigned long long*>(h->d_err + 2);
    launch_accuracy(m, n, C, ldc, hi, lo, reinterpret_cast<unsigned int*>(h->d_err + 1), cnt, h->stream);
    ++h->launches;
    unsigned int out[3] = {0, 0, 0};
    OZ2_CUDA(h, cudaMemcpyAsync(out, h->d_err + 1, sizeof out, cudaMemcpyDeviceToHost, h->stream));
    OZ2_CUDA(h, cudaStreamSynchronize(h->stream));
    float f;
    std::memcpy(&f, &out[0], sizeof f);
    unsigned long long c;
    std::memcpy(&c, &out[1], sizeof c);
    *max_ulp = f;
    *correctly_rounded = static_cast<int64_t>(c);
    return OZ2_OK;
}

int oz2_kernel_launches(oz2_handle h, int64_t* out) {
    if (!h || !out) return fail(h, OZ2_EINVAL, "oz2: null argument");
    *out = h->launches;
    return OZ2_OK;
}

int oz2_set_graph_mode(oz2_handle h, int enable) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    h->graph_mode = enable != 0;
    if (!h->graph_mode) drop_graphs(h);
    return OZ2_OK;
}

int oz2_set_gemm_config(oz2_handle h, int bn, int group_j, int ctas) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    if (bn == 0) {
        h->has_forced = false;
        drop_graphs(h);
        return OZ2_OK;
    }
    if ((bn != 128 && bn != 256) || group_j < 1 || ctas < 0)
        return fail(h, OZ2_EINVAL, "oz2: gemm config: bn must be 128 or 256, group_j >= 1, ctas >= 0");
    h->forced = GemmConfig{bn, group_j, ctas};
    h->has_forced = true;
    drop_graphs(h);
    return OZ2_OK;
}

int oz2_get_gemm_config(oz2_handle h, int* out3) {
    if (!h || !out3) return fail(h, OZ2_EINVAL, "oz2: null argument");
    out3[0] = h->last_cfg.bn;
    out3[1] = h->last_cfg.group_j;
    out3[2] = h->last_cfg.ctas;
    return OZ2_OK;
}

// Times the grouped call's GEMM phase under each candidate configuration (tile width along i,
// raster group, CTA count) on the caller's problems and keeps the fastest for problem sets of
// the same shapes. Runs the problems (C is written) once per candidate plus once to warm up.
int oz2_autotune_grouped(oz2_handle h, int count, const oz2_dgemm_problem* problems, int* out3) {
    if (!h) return fail(nullptr, OZ2_EINVAL, "oz2: null handle");
    std::vector<Prob> probs;
    int st = validate_grouped(h, count, problems, probs);
    if (st) return st;
    if (probs.empty()) return fail(h, OZ2_EINVAL, "oz2: nothing to tune");
    std::vector<const Prob*> bp;
    for (auto& p : probs) bp.push_back(&p);
    const bool had_forced = h->has_forced, had_graph = h->graph_mode, had_prof = h->profiling;
    const GemmConfig saved = h->forced;
    h->graph_mode = false;
    h->profiling = true;
    std::vector<GemmConfig> cands;
    for (int bn : {256, 128})
        for (int gj : {4, 8, 16, 32}) cands.push_back(GemmConfig{bn, gj, 0});
    GemmConfig best = heuristic_config(bp);
    double best_ms = std::numeric_limits<double>::infinity();
    h->forced = best;
    h->has_forced = true;
    if ((st = run_grouped(h, probs))) goto done;  // warm-up
    for (const GemmConfig& c : cands) {
        h->forced = c;
        double total = 0;
        for (int rep = 0; rep < 2; ++rep) {
            h->marks.clear();
            h->pool_used = 0;
            if ((st = run_grouped(h, probs))) goto done;
            double v[4];
            if ((st = oz2_stage_times(h, v))) goto done;
            total += v[2];
        }
        if (total < best_ms) {
            best_ms = total;
            best = c;
        }
    }
    h->tuned[shape_signature(bp)] = best;
    drop_graphs(h);
    if (out3) {
        out3[0] = best.bn;
        out3[1] = best.group_j;
        out3[2] = best.ctas;
    }
done:
    h->has_forced = had_forced;
    h->forced = saved;
    h->graph_mode = had_graph;
    h->profiling = had_prof;
    return st;
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
    drop_graphs(h);
    cudaFree(h->ws);
    h->ws = nullptr;
    h->ws_size = 0;
    ++h->ws_gen;
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

int oz2_adaptive_stage_times(oz2_handle h, double* out2) {
    if (!h || !out2) return fail(h, OZ2_EINVAL, "oz2: null argument");
    out2[0] = out2[1] = 0.0;
    if (!h->profiling) return OZ2_OK;
    out2[1] = h->native_ms;
    if (h->marks.empty()) return OZ2_OK;
    OZ2_CUDA(h, cudaEventSynchronize(h->marks.back().second));
    for (size_t i = 1; i < h->marks.size(); ++i) {
        const int stg = h->marks[i].first;
        if (stg != kProbe && stg != kNative) continue;
        float ms = 0.0f;
        OZ2_CUDA(h, cudaEventElapsedTime(&ms, h->marks[i - 1].second, h->marks[i].second));
        out2[stg - kProbe] += ms;
    }
    return OZ2_OK;
}

int oz2_adaptive_gemm_bytes(oz2_handle h, int64_t* out3) {
    if (!h || !out3) return fail(h, OZ2_EINVAL, "oz2: null argument");
    for (int i = 0; i < 3; ++i) out3[i] = h->gbytes[i];
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

int oz2_set_failure_test(int64_t wait_limit_ns, int stall_mma) {
    if (wait_limit_ns < 0) return fail(nullptr, OZ2_EINVAL, "oz2: negative wait limit");
    set_gemm_failure_test(static_cast<uint64_t>(wait_limit_ns), stall_mma);
    return OZ2_OK;
}

int oz2_set_split_kernel(int kind) {
    if (kind != 0 && kind != 1) return fail(nullptr, OZ2_EINVAL, "oz2: split kernel must be 0 (dp4a) or 1 (tensor core)");
    set_split_path(kind);
    return OZ2_OK;
}

int oz2_set_crt_kernel(int kind) {
    if (kind < 0 || kind > 2) return fail(nullptr, OZ2_EINVAL, "oz2: CRT kernel must be 0 (dp2a), 1 (tensor core) or 2 (auto)");
    set_crt_path(kind);
    return OZ2_OK;
}

int oz2_set_scale_fusion(int on) {
    set_scale_fusion(on);
    return OZ2_OK;
}

int oz2_set_crt_fusion(int on) {
    set_crt_fusion(on);
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
