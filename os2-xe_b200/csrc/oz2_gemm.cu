// oz2_gemm.cu - the s (3s for ZGEMM) INT8 products of the Ozaki-II path on the tcgen05 tensor
// cores, with the reduction modulo m_t fused into the epilogue.
//
// Replaces the reference's oneMKL int8 gemm_batch (src/ozaki2_gpu.hpp:1029-1040, :883-890) and
// the int32 -> residue step of its CRT kernel (rep_i32 / gemm_residue :305-307, :590-601):
// instead of s int32 planes (4 bytes per entry) the kernel writes one uint8 residue c mod m_t
// per entry, so the CRT phase reads 1 byte per entry and modulus.
//
// Persistent kernel, one CTA per SM, 6 warps:
//   warp 0   producer: 1-D bulk copies of pre-tiled 16 KiB plane tiles into a 4-stage ring
//   warp 1   MMA issuer: tcgen05.mma kind::i8, M=128 (columns j of C), N=256 (rows i of C),
//            K=32 per instruction, int32 accumulators in TMEM (2 x 256 columns, double buffer)
//   warps 2-5 epilogue: tcgen05.ld 32 lanes x 32 columns, c mod m_t, 32 residue bytes per
//            thread and chunk stored to residue plane row j (i contiguous)
// Every mbarrier wait is time-bounded; on expiry the kernel records an error code, drains its
// in-flight copies and MMAs, frees TMEM and returns.
#include <algorithm>
#include <cstdio>

#include "oz2_kernels.cuh"
#include "oz2_ptx.cuh"

namespace oz2 {
namespace {

constexpr int kStages = 4;
constexpr int kStageJ = kGemmJ * kTileK;              // 16 KiB
constexpr int kStageI = kGemmI * kTileK;              // 32 KiB
constexpr int kStageBytes = kStageJ + kStageI;       // 48 KiB
constexpr int kGroupJ = 16;                          // raster: 16 column tiles share the row panels
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kIdesc = dev::idesc_i8(kGemmJ, kGemmI);
constexpr int kBarBytes = 256;
constexpr int kSmemBytes = 1024 + kStages * kStageBytes + kBarBytes;

struct GemmParams {
    const int8_t* planes_i;
    const int8_t* planes_j;
    uint8_t* resid;
    int64_t pstride_i, pstride_j, rstride, ldr, m, n, kb_total, kb0, kb1;
    int64_t tiles, jobs;
    int tiles_i, tiles_j, s, accumulate;
    int* err;
    uint32_t mod_m[kMaxModuli], mod_mu[kMaxModuli], mod_kneg[kMaxModuli];
};

struct Job {
    int gt;  // group * s + modulus
    int ti, tj;
};
__device__ __forceinline__ Job decode(const GemmParams& P, int64_t job) {
    Job J;
    J.gt = static_cast<int>(job / P.tiles);
    const int64_t tile = job - static_cast<int64_t>(J.gt) * P.tiles;
    const int64_t per_grp = static_cast<int64_t>(kGroupJ) * P.tiles_i;
    const int64_t grp = tile / per_grp, rem = tile - grp * per_grp;
    const int first_j = static_cast<int>(grp) * kGroupJ;
    const int gj = min(kGroupJ, P.tiles_j - first_j);
    J.tj = first_j + static_cast<int>(rem % gj);
    J.ti = static_cast<int>(rem / gj);
    return J;
}

__global__ void __launch_bounds__(192, 1) gemm_i8_modm_kernel(const __grid_constant__ GemmParams P) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t{1023});
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
    // barriers: full[kStages] empty[kStages] acc_full[2] acc_empty[2] drain
    const uint32_t bar0 = dev::smem_addr(bars);
    auto full = [&](int i) { return bar0 + 8u * i; };
    auto empty = [&](int i) { return bar0 + 8u * (kStages + i); };
    auto acc_full = [&](int a) { return bar0 + 8u * (2 * kStages + a); };
    auto acc_empty = [&](int a) { return bar0 + 8u * (2 * kStages + 2 + a); };
    const uint32_t drain = bar0 + 8u * (2 * kStages + 4);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 5);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int i = 0; i < kStages; ++i) {
            dev::mbar_init(full(i), 1);
            dev::mbar_init(empty(i), 1);
        }
        for (int a = 0; a < 2; ++a) {
            dev::mbar_init(acc_full(a), 1);
            dev::mbar_init(acc_empty(a), 4);
        }
        dev::mbar_init(drain, 1);
        *abort_flag = 0;
        dev::fence_barrier_init();
    }
    if (warp == 1) {
        dev::tmem_alloc(dev::smem_addr(tmem_slot), kTmemCols);
        dev::tmem_relinquish();
    }
    dev::tc_fence_before();
    __syncthreads();
    dev::tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const int64_t nprog = gridDim.x;
    const int64_t row_block = P.kb_total * kTileBytes;

    if (warp == 0) {
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            uint32_t issued_mask = 0, issued_phase = 0;
            bool ok = true;
            for (int64_t job = blockIdx.x; ok && job < P.jobs; job += nprog) {
                const Job J = decode(P, job);
                const int8_t* srcJ = P.planes_j + J.gt * P.pstride_j + J.tj * row_block;
                const int8_t* srcI = P.planes_i + J.gt * P.pstride_i + (2 * static_cast<int64_t>(J.ti)) * row_block;
                for (int64_t kb = P.kb0; kb < P.kb1; ++kb) {
                    if (!dev::mbar_wait(empty(stage), phase ^ 1u, abort_flag, P.err, dev::kErrTimeoutEmpty)) {
                        ok = false;
                        break;
                    }
                    const uint32_t sJ = dev::smem_addr(smem + stage * kStageBytes);
                    const uint32_t sI = sJ + kStageJ;
                    dev::mbar_arrive_expect_tx(full(stage), kStageBytes);
                    dev::bulk_load(sJ, srcJ + kb * kTileBytes, kTileBytes, full(stage));
                    dev::bulk_load(sI, srcI + kb * kTileBytes, kTileBytes, full(stage));
                    dev::bulk_load(sI + kTileBytes, srcI + row_block + kb * kTileBytes, kTileBytes, full(stage));
                    issued_mask |= 1u << stage;
                    issued_phase = (issued_phase & ~(1u << stage)) | (phase << stage);
                    if (++stage == kStages) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
            }
            if (!ok) {  // let every copy that was issued land before the CTA exits
                for (int i = 0; i < kStages; ++i)
                    if (issued_mask & (1u << i)) dev::mbar_wait_drain(full(i), (issued_phase >> i) & 1u);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            bool ok = true, issued = false;
            int local = 0;
            for (int64_t job = blockIdx.x; ok && job < P.jobs; job += nprog, ++local) {
                const int acc = local & 1;
                const uint32_t use = static_cast<uint32_t>(local >> 1);
                if (!dev::mbar_wait(acc_empty(acc), (use & 1u) ^ 1u, abort_flag, P.err, dev::kErrTimeoutAccEmpty)) {
                    ok = false;
                    break;
                }
                dev::tc_fence_after();
                const uint32_t d_tmem = tmem_base + static_cast<uint32_t>(acc) * kGemmI;
                for (int64_t kb = P.kb0; kb < P.kb1; ++kb) {
                    if (!dev::mbar_wait(full(stage), phase, abort_flag, P.err, dev::kErrTimeoutFull)) {
                        ok = false;
                        break;
                    }
                    dev::tc_fence_after();
                    const uint32_t sJ = dev::smem_addr(smem + stage * kStageBytes);
                    const uint32_t sI = sJ + kStageJ;
#pragma unroll
                    for (int kk = 0; kk < kTileK / 32; ++kk) {
                        dev::mma_i8(d_tmem, dev::sw128_kmajor_desc(sJ + kk * 32), dev::sw128_kmajor_desc(sI + kk * 32),
                                    kIdesc, (kb > P.kb0 || kk > 0) ? 1u : 0u);
                    }
                    issued = true;
                    dev::tc_commit(empty(stage));
                    if (++stage == kStages) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
                if (!ok) break;
                dev::tc_commit(acc_full(acc));
            }
            if (!ok && issued) {  // wait until every MMA issued so far has completed
                dev::tc_commit(drain);
                dev::mbar_wait_drain(drain, 0);
            }
        }
    } else {
        const int quarter = warp & 3;  // TMEM lanes this warp may access
        int local = 0;
        for (int64_t job = blockIdx.x; job < P.jobs; job += nprog, ++local) {
            const int acc = local & 1;
            const uint32_t use = static_cast<uint32_t>(local >> 1);
            int ok = 1;
            if (lane == 0) ok = dev::mbar_wait(acc_full(acc), use & 1u, abort_flag, P.err, dev::kErrTimeoutAccFull);
            ok = __shfl_sync(0xFFFFFFFFu, ok, 0);
            if (!ok) break;
            dev::tc_fence_after();
            const Job J = decode(P, job);
            const int t = J.gt % P.s;
            const uint32_t m = P.mod_m[t], mu = P.mod_mu[t], kneg = P.mod_kneg[t];
            const int64_t j = static_cast<int64_t>(J.tj) * kGemmJ + quarter * 32 + lane;
            uint8_t* row = P.resid + J.gt * P.rstride + j * P.ldr;
            const uint32_t taddr = tmem_base + (static_cast<uint32_t>(quarter * 32) << 16) +
                                   static_cast<uint32_t>(acc) * kGemmI;
#pragma unroll 1
            for (int c = 0; c < kGemmI / 32; ++c) {
                uint32_t v[32];
                dev::tmem_load_32x32(taddr + c * 32, v);
                dev::tmem_load_wait();
                const int64_t i0 = static_cast<int64_t>(J.ti) * kGemmI + c * 32;
                if (j < P.n && i0 < P.m) {
                    uint32_t w[8];
                    uint4 old0 = make_uint4(0, 0, 0, 0), old1 = old0;
                    if (P.accumulate) {
                        old0 = *reinterpret_cast<const uint4*>(row + i0);
                        old1 = *reinterpret_cast<const uint4*>(row + i0 + 16);
                    }
                    const uint32_t ow[8] = {old0.x, old0.y, old0.z, old0.w, old1.x, old1.y, old1.z, old1.w};
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        uint32_t word = 0;
#pragma unroll
                        for (int b = 0; b < 4; ++b) {
                            const uint32_t u = v[4 * q + b] + 0x80000000u;  // int32 c + 2^31
                            const uint32_t qq = __umulhi(u, mu);
                            uint32_t r = u - qq * m;
                            r = min(r, r - m);    // (c + 2^31) mod m
                            r += kneg;
                            r = min(r, r - m);    // c mod m
                            if (P.accumulate) {
                                r += (ow[q] >> (8 * b)) & 0xFFu;
                                r = min(r, r - m);
                            }
                            word |= r << (8 * b);
                        }
                        w[q] = word;
                    }
                    *reinterpret_cast<uint4*>(row + i0) = make_uint4(w[0], w[1], w[2], w[3]);
                    *reinterpret_cast<uint4*>(row + i0 + 16) = make_uint4(w[4], w[5], w[6], w[7]);
                }
            }
            dev::tc_fence_before();
            __syncwarp();
            if (lane == 0) dev::mbar_arrive(acc_empty(acc));
        }
    }
    __syncwarp();
    dev::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        dev::tc_fence_after();
        dev::tmem_dealloc(tmem_base, kTmemCols);
    }
}

}  // namespace

void launch_gemm(const GemmArgs& a, int num_sms, cudaStream_t st) {
    GemmParams P{};
    P.planes_i = a.planes_i;
    P.planes_j = a.planes_j;
    P.resid = a.resid;
    P.pstride_i = a.pstride_i;
    P.pstride_j = a.pstride_j;
    P.rstride = a.rstride;
    P.ldr = a.ldr;
    P.m = a.m;
    P.n = a.n;
    P.kb_total = a.kb_total;
    P.kb0 = a.kb0;
    P.kb1 = a.kb1;
    P.tiles_i = static_cast<int>(ceil_div(a.m, kGemmI));
    P.tiles_j = static_cast<int>(ceil_div(a.n, kGemmJ));
    P.tiles = static_cast<int64_t>(P.tiles_i) * P.tiles_j;
    P.jobs = P.tiles * a.groups * a.s;
    P.s = a.s;
    P.accumulate = a.accumulate;
    P.err = a.err;
    for (int t = 0; t < a.s; ++t) {
        P.mod_m[t] = a.mc[t].m;
        P.mod_mu[t] = a.mc[t].mu;
        P.mod_kneg[t] = a.mc[t].kneg;
    }
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(gemm_i8_modm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
        attr_set = true;
    }
    const int64_t grid = std::min<int64_t>(num_sms, P.jobs);
    if (grid <= 0) return;
    gemm_i8_modm_kernel<<<static_cast<unsigned>(grid), 192, kSmemBytes, st>>>(P);
}

}  // namespace oz2
