// oz2_gemm.cu - the s (3s for ZGEMM) INT8 products of the Ozaki-II path on the tcgen05 tensor
// cores, with the reduction modulo m_t fused into the epilogue.
//
// Replaces the reference's oneMKL int8 gemm_batch (src/ozaki2_gpu.hpp:1029-1040, :883-890) and
// the int32 -> residue step of its CRT kernel (rep_i32 / gemm_residue :305-307, :590-601):
// instead of s int32 planes (4 bytes per entry) the kernel writes one uint8 residue c mod m_t
// per entry, so the CRT phase reads 1 byte per entry and modulus.
//
// Persistent kernel over a table of problems (one emulated GEMM, or a group of them), one CTA
// per SM, 10 warps:
//   warp 0   producer: 1-D bulk copies of pre-tiled 16 KiB plane tiles into a 4-stage ring
//   warp 1   MMA issuer: tcgen05.mma kind::i8, M=128 (columns j of C), N=BN (rows i of C,
//            BN = 256 or 128), K=32 per instruction, int32 accumulators in TMEM (2 x BN
//            columns, double buffer); k beyond 130944 runs as chunks inside one job, each chunk
//            adding its residues to the previous ones mod m
//   warps 2-9 epilogue, two per TMEM lane quarter, each half of the BN columns: tcgen05.ld
//            32 lanes x 32 columns (the next load in flight during the arithmetic), c mod m_t
//            as (c + m ceil(2^31/m)) mod m with one Barrett step, 32 residue bytes per thread
//            and chunk: a warp's 32 rows j x 32 columns i form one contiguous kilobyte of the
//            residue plane (layout in oz2_kernels.cuh)
// Every mbarrier wait is time-bounded; on expiry the kernel records an error code, drains its
// in-flight copies and MMAs, frees TMEM and returns.
#include <algorithm>
#include <atomic>
#include <cstdio>

#include "oz2_crt_math.cuh"
#include "oz2_kernels.cuh"
#include "oz2_ptx.cuh"

namespace oz2 {
namespace {

constexpr uint32_t kBarBytes = 256;
constexpr int kEpiWarps = 8;                       // two per TMEM lane quarter (four measured slower)
constexpr int kEpiParts = kEpiWarps / 4;           // column ranges of the accumulator
constexpr int kGemmThreads = 64 + 32 * kEpiWarps;  // producer, MMA issuer, epilogue

template <int BN>
struct Cfg {
    static constexpr int kStageJ = kGemmJ * kTileK;       // 16 KiB
    static constexpr int kStageI = BN * kTileK;           // 32 KiB (BN 256) / 16 KiB (BN 128)
    static constexpr int kStageBytes = kStageJ + kStageI;
    static constexpr int kStages = BN == 256 ? 4 : 6;
    static constexpr uint32_t kTmemCols = 2 * BN;         // two accumulators
    static constexpr uint32_t kIdesc = dev::idesc_i8(kGemmJ, BN);
    static constexpr int kSmemBytes = 1024 + kStages * kStageBytes + kBarBytes;
};

struct GemmParams {
    const GemmItem* items;
    int count;
    int group_j;
    int64_t jobs;
    int* err;
    uint64_t wait_ns;  // limit of every bounded mbarrier wait
    int stall;         // failure-path test: the MMA issuer issues nothing, so the waits run out
    CrtConst cc;       // kKindCrt: the plan's CRT constants (all items of the launch share the plan)
};

struct Job {
    const GemmItem* I;
    int gt;  // group * s + modulus
    int ti, tj;
    int64_t nch;  // k chunks
};
// per_tile: the job is a tile and runs every modulus (kKindCrt); otherwise (group, modulus, tile)
__device__ __forceinline__ Job decode(const GemmParams& P, int64_t job, bool per_tile = false) {
    int lo = 0, hi = P.count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (P.items[mid].job0 <= job) lo = mid;
        else hi = mid - 1;
    }
    Job J;
    J.I = P.items + lo;
    // 32-bit arithmetic: an item's jobs (groups * s * tiles) are bounded by its residue planes,
    // s m n bytes of device memory, so they stay far below 2^32 (one 64-bit division costs
    // several times a 32-bit one, and every warp decodes every job)
    const uint32_t local = static_cast<uint32_t>(job - J.I->job0);
    const uint32_t tiles = static_cast<uint32_t>(J.I->tiles);
    const uint32_t gt = per_tile ? 0u : local / tiles;
    J.gt = static_cast<int>(gt);
    const uint32_t tile = local - gt * tiles;
    const uint32_t tiles_i = static_cast<uint32_t>(J.I->tiles_i), tiles_j = static_cast<uint32_t>(J.I->tiles_j);
    const uint32_t group_j = static_cast<uint32_t>(P.group_j);
    const uint32_t per_grp = group_j * tiles_i;
    const uint32_t grp = tile / per_grp, rem = tile - grp * per_grp;
    const uint32_t first_j = grp * group_j;
    const uint32_t gj = min(group_j, tiles_j - first_j);
    const uint32_t qj = rem / gj;
    J.tj = static_cast<int>(first_j + (rem - qj * gj));
    J.ti = static_cast<int>(qj);
    J.nch = (J.I->kb_total + kChunkKB - 1) / kChunkKB;
    return J;
}

// KIND: kKindResidue the Ozaki-II GEMM (int8 planes, residues mod m); kKindOz1 the Ozaki Scheme I
// baseline (job t = digit pair, int64 atomic sums per anti-diagonal instead of residues);
// kKindCert the certificate (bf16 planes of scaled magnitudes, kind::f16 MMAs, the largest
// (R'_i + S'_j) / G_ij and 1 / G_ij per adaptive tile instead of residues)
// kKindCrt the Ozaki-II GEMM with the CRT in the epilogue (a job is a tile and all its s <= 8
// moduli: each modulus's residues go to tensor memory as packed bytes, columns 2 BN + 128 h + 16 t
// + w for epilogue half h, modulus t and word w; after the last modulus the epilogue reconstructs
// its 64 entries per lane and writes C)
constexpr int kKindResidue = 0, kKindOz1 = 1, kKindCert = 2, kKindCrt = 3;

template <int BN, int KIND>
__global__ void __launch_bounds__(kGemmThreads, 1) gemm_i8_modm_kernel(const __grid_constant__ GemmParams P) {
    constexpr bool OZ1 = KIND == kKindOz1, CERT = KIND == kKindCert, CRTF = KIND == kKindCrt;
    static_assert(!CRTF || BN == 128, "the fused CRT keeps its residues beside two 128-column accumulators");
    using C = Cfg<BN>;
    constexpr uint32_t kTmemCols = CRTF ? 512u : C::kTmemCols;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t{1023});
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + C::kStages * C::kStageBytes);
    // barriers: full[kStages] empty[kStages] acc_full[2] acc_empty[2] drain
    const uint32_t bar0 = dev::smem_addr(bars);
    auto full = [&](int i) { return bar0 + 8u * i; };
    auto empty = [&](int i) { return bar0 + 8u * (C::kStages + i); };
    auto acc_full = [&](int a) { return bar0 + 8u * (2 * C::kStages + a); };
    auto acc_empty = [&](int a) { return bar0 + 8u * (2 * C::kStages + 2 + a); };
    const uint32_t drain = bar0 + 8u * (2 * C::kStages + 4);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * C::kStages + 5);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int i = 0; i < C::kStages; ++i) {
            dev::mbar_init(full(i), 1);
            dev::mbar_init(empty(i), 1);
        }
        for (int a = 0; a < 2; ++a) {
            dev::mbar_init(acc_full(a), 1);
            dev::mbar_init(acc_empty(a), kEpiWarps);
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

    if (warp == 0) {
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            uint32_t issued_mask = 0, issued_phase = 0;
            bool ok = true;
            for (int64_t job = blockIdx.x; ok && job < P.jobs; job += nprog) {
                const Job J = decode(P, job, CRTF);
                const int64_t kb_total = J.I->kb_total, row_block = kb_total * kTileBytes;
                const int nt = CRTF ? J.I->s : 1;
                for (int tt = 0; ok && tt < nt; ++tt) {
                const int gt = CRTF ? tt : J.gt;
                const int pj = OZ1 ? J.I->pair_b[gt] : gt, pi = OZ1 ? J.I->pair_a[gt] : gt;
                const int8_t* srcJ = J.I->planes_j + pj * J.I->pstride_j + J.tj * row_block;
                const int8_t* srcI = J.I->planes_i + pi * J.I->pstride_i + (static_cast<int64_t>(J.ti) * (BN / 128)) * row_block;
                for (int64_t kb = 0; ok && kb < kb_total; ++kb) {
                    if (!dev::mbar_wait(empty(stage), phase ^ 1u, abort_flag, P.err, dev::kErrTimeoutEmpty,
                                         P.wait_ns)) {
                        ok = false;
                        break;
                    }
                    const uint32_t sJ = dev::smem_addr(smem + stage * C::kStageBytes);
                    const uint32_t sI = sJ + C::kStageJ;
                    dev::mbar_arrive_expect_tx(full(stage), C::kStageBytes);
                    dev::bulk_load(sJ, srcJ + kb * kTileBytes, kTileBytes, full(stage));
                    dev::bulk_load(sI, srcI + kb * kTileBytes, kTileBytes, full(stage));
                    if (BN == 256) dev::bulk_load(sI + kTileBytes, srcI + row_block + kb * kTileBytes, kTileBytes, full(stage));
                    issued_mask |= 1u << stage;
                    issued_phase = (issued_phase & ~(1u << stage)) | (phase << stage);
                    if (++stage == C::kStages) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
                }
            }
            if (!ok) {  // let every copy that was issued land before the CTA exits
                for (int i = 0; i < C::kStages; ++i)
                    if (issued_mask & (1u << i)) dev::mbar_wait_drain(full(i), (issued_phase >> i) & 1u);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            bool ok = !P.stall, issued = false;
            int local = 0;  // (job, chunk) pairs processed: selects the accumulator
            for (int64_t job = blockIdx.x; ok && job < P.jobs; job += nprog) {
                const Job J = decode(P, job, CRTF);
                const int64_t kb_total = J.I->kb_total;
                const int nt = CRTF ? J.I->s : 1;
                for (int tt = 0; ok && tt < nt; ++tt)
                for (int64_t c = 0; ok && c < J.nch; ++c, ++local) {
                    const int acc = local & 1;
                    const uint32_t use = static_cast<uint32_t>(local >> 1);
                    if (!dev::mbar_wait(acc_empty(acc), (use & 1u) ^ 1u, abort_flag, P.err, dev::kErrTimeoutAccEmpty,
                                         P.wait_ns)) {
                        ok = false;
                        break;
                    }
                    dev::tc_fence_after();
                    const uint32_t d_tmem = tmem_base + static_cast<uint32_t>(acc) * BN;
                    const int64_t kb0 = c * kChunkKB, kb1 = min(kb_total, kb0 + kChunkKB);
                    for (int64_t kb = kb0; kb < kb1; ++kb) {
                        if (!dev::mbar_wait(full(stage), phase, abort_flag, P.err, dev::kErrTimeoutFull,
                                             P.wait_ns)) {
                            ok = false;
                            break;
                        }
                        dev::tc_fence_after();
                        const uint32_t sJ = dev::smem_addr(smem + stage * C::kStageBytes);
                        const uint32_t sI = sJ + C::kStageJ;
#pragma unroll
                        for (int kk = 0; kk < kTileK / 32; ++kk) {
                            if constexpr (CERT)
                                dev::mma_bf16(d_tmem, dev::sw128_kmajor_desc(sJ + kk * 32),
                                              dev::sw128_kmajor_desc(sI + kk * 32), dev::idesc_bf16(kGemmJ, BN),
                                              (kb > kb0 || kk > 0) ? 1u : 0u);
                            else
                                dev::mma_i8(d_tmem, dev::sw128_kmajor_desc(sJ + kk * 32),
                                            dev::sw128_kmajor_desc(sI + kk * 32), C::kIdesc,
                                            (kb > kb0 || kk > 0) ? 1u : 0u);
                        }
                        issued = true;
                        dev::tc_commit(empty(stage));
                        if (++stage == C::kStages) {
                            stage = 0;
                            phase ^= 1u;
                        }
                    }
                    if (!ok) break;
                    dev::tc_commit(acc_full(acc));
                }
            }
            if (!ok && issued) {  // wait until every MMA issued so far has completed
                dev::tc_commit(drain);
                dev::mbar_wait_drain(drain, 0);
            }
        }
    } else {
        const int quarter = warp & 3;           // TMEM lanes this warp may access
        const int half = (warp - 2) >> 2;       // which part of the BN columns
        constexpr int kChunks = BN / 32 / kEpiParts;  // 32-column chunks per warp
        int local = 0;
        bool ok = true;
        for (int64_t job = blockIdx.x; ok && job < P.jobs; job += nprog) {
            const Job J = decode(P, job, CRTF);
            const int nt = CRTF ? J.I->s : 1;
            for (int tt = 0; ok && tt < nt; ++tt) {
            const int t = CRTF ? tt : J.gt % J.I->s;
            constexpr bool RES = KIND == kKindResidue || CRTF;
            const uint32_t m = RES ? J.I->mod_m[t] : 1u, mu = RES ? J.I->mod_mu[t] : 0u,
                           kbias = RES ? J.I->mod_kbias[t] : 0u;
            // at most kExactKB k-blocks (one chunk): |c| <= kExactSum, so u = c + kbias30 < 2^31 and
            // the multiply-high quotient is exact; otherwise Barrett with one correction step
            const bool exact = RES && J.I->kb_total <= kExactKB;
            const uint32_t kbias30 = RES ? J.I->mod_kbias30[t] : 0u, mx31 = RES ? J.I->mod_mx31[t] : 0u;
            const uint32_t mxs = RES ? J.I->mod_mxs[t] : 7u;
            const int64_t j = static_cast<int64_t>(J.tj) * kGemmJ + quarter * 32 + lane;
            const int64_t mm = J.I->m, nn = J.I->n;
            uint8_t* rowj = RES && !CRTF ? J.I->resid + J.gt * J.I->rstride + j * 32 : nullptr;  // + (i / 32) * 32 n
            // certificate: this lane's column sum (zero for a padding column or an all-zero column,
            // whose entries are skipped)
            const float sj = CERT && j < nn ? static_cast<float>(J.I->cert_sb[j]) : 0.0f;
            for (int64_t c = 0; c < J.nch; ++c, ++local) {
                const int acc = local & 1;
                const uint32_t use = static_cast<uint32_t>(local >> 1);
                int w_ok = 1;
                if (lane == 0) w_ok = dev::mbar_wait(acc_full(acc), use & 1u, abort_flag, P.err, dev::kErrTimeoutAccFull,
                                                  P.wait_ns);
                w_ok = __shfl_sync(0xFFFFFFFFu, w_ok, 0);
                if (!w_ok) {
                    ok = false;
                    break;
                }
                dev::tc_fence_after();
                const bool accumulate = c > 0;
                const uint32_t taddr = tmem_base + (static_cast<uint32_t>(quarter * 32) << 16) +
                                       static_cast<uint32_t>(acc) * BN + static_cast<uint32_t>(half * kChunks * 32);
                uint32_t v[2][32];
                dev::tmem_load_32x32(taddr, v[0]);
                dev::tmem_load_wait();
#pragma unroll
                for (int cc = 0; cc < kChunks; ++cc) {
                    uint32_t(&cur)[32] = v[cc & 1];
                    // the next chunk's load is in flight during this chunk's arithmetic
                    if (cc + 1 < kChunks) dev::tmem_load_32x32(taddr + (cc + 1) * 32, v[(cc + 1) & 1]);
                    const int64_t i0 = static_cast<int64_t>(J.ti) * BN + (half * kChunks + cc) * 32;
                    uint8_t* blk = rowj + (i0 >> 5) * (32 * nn);  // this chunk's 32 bytes of row j
                    if constexpr (CERT) {
                        // the warp's 32 lanes are 32 consecutive j of one adaptive tile column
                        // (cert_tile is a multiple of 128), its 32 columns i0.. one tile row
                        float q1 = 0.0f, q2 = 0.0f;
                        if (sj > 0.0f) {
#pragma unroll
                            for (int b = 0; b < 32; ++b) {
                                const int64_t i = i0 + b;
                                const float ri = i < mm ? static_cast<float>(__ldg(J.I->cert_ra + i)) : 0.0f;
                                if (ri > 0.0f) {
                                    const float g = __uint_as_float(cur[b]);
                                    if (g > 0.0f) {
                                        const float rg = __fdividef(1.0f, g);  // within 2 ulp
                                        q1 = fmaxf(q1, (ri + sj) * rg);
                                        q2 = fmaxf(q2, rg);
                                    } else {
                                        q1 = q2 = __int_as_float(0x7F800000);
                                    }
                                }
                            }
                        }
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) {
                            q1 = fmaxf(q1, __shfl_xor_sync(0xFFFFFFFFu, q1, o));
                            q2 = fmaxf(q2, __shfl_xor_sync(0xFFFFFFFFu, q2, o));
                        }
                        if (lane == 0 && i0 < mm && q1 > 0.0f) {
                            const int64_t T = J.I->cert_tile;
                            const int64_t jw = static_cast<int64_t>(J.tj) * kGemmJ + quarter * 32;
                            unsigned int* slot = J.I->cert_q + 2 * ((jw / T) * J.I->cert_na + i0 / T);
                            atomicMax(slot, __float_as_uint(q1));  // non-negative floats order as their bits
                            atomicMax(slot + 1, __float_as_uint(q2));
                        }
                    } else if constexpr (OZ1) {
                        if (j < nn) {  // a warp's lanes are 32 consecutive j: 256 contiguous bytes per row i
                            unsigned long long* dst = reinterpret_cast<unsigned long long*>(
                                J.I->acc + J.I->pair_d[J.gt] * J.I->acc_plane + j);
                            const int64_t ld = J.I->acc_ld;
#pragma unroll
                            for (int b = 0; b < 32; ++b)
                                if (i0 + b < mm)
                                    atomicAdd(dst + (i0 + b) * ld, static_cast<unsigned long long>(
                                                                       static_cast<long long>(static_cast<int32_t>(cur[b]))));
                        }
                    } else if constexpr (CRTF) {
                        // residues of this modulus as packed bytes into tensor memory (every lane
                        // and chunk: padding entries are never read back)
                        uint32_t w[8];
#pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            uint32_t r4[4];
#pragma unroll
                            for (int b = 0; b < 4; ++b) {
                                const uint32_t u = cur[4 * q + b] + kbias30;
                                r4[b] = u - (__umulhi(u, mx31) >> mxs) * m;
                            }
                            w[q] = __byte_perm(__byte_perm(r4[0], r4[1], 0x0040), __byte_perm(r4[2], r4[3], 0x0040), 0x5410);
                        }
                        dev::tmem_store_32x8(tmem_base + (static_cast<uint32_t>(quarter * 32) << 16) +
                                                 static_cast<uint32_t>(2 * BN + 128 * half + 16 * tt + 8 * cc),
                                             w);
                    } else if (exact) {
                        if (j < nn && i0 < mm) {
                            uint32_t w[8];
#pragma unroll
                            for (int q = 0; q < 8; ++q) {
                                uint32_t r4[4];
#pragma unroll
                                for (int b = 0; b < 4; ++b) {
                                    const uint32_t u = cur[4 * q + b] + kbias30;  // in [0, 2^31)
                                    r4[b] = u - (__umulhi(u, mx31) >> mxs) * m;  // in [0, m)
                                }
                                w[q] = __byte_perm(__byte_perm(r4[0], r4[1], 0x0040),
                                                   __byte_perm(r4[2], r4[3], 0x0040), 0x5410);
                            }
                            *reinterpret_cast<uint4*>(blk) = make_uint4(w[0], w[1], w[2], w[3]);
                            *reinterpret_cast<uint4*>(blk + 16) = make_uint4(w[4], w[5], w[6], w[7]);
                        }
                    } else if (j < nn && i0 < mm) {
                        uint32_t ow[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                        if (accumulate) {
                            const uint4 o0 = *reinterpret_cast<const uint4*>(blk);
                            const uint4 o1 = *reinterpret_cast<const uint4*>(blk + 16);
                            ow[0] = o0.x; ow[1] = o0.y; ow[2] = o0.z; ow[3] = o0.w;
                            ow[4] = o1.x; ow[5] = o1.y; ow[6] = o1.z; ow[7] = o1.w;
                        }
                        uint32_t w[8];
#pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            uint32_t r4[4];
#pragma unroll
                            for (int b = 0; b < 4; ++b) {
                                const uint32_t u = cur[4 * q + b] + kbias;  // c + m ceil(2^31/m), in [0, 2^32)
                                uint32_t r = u - __umulhi(u, mu) * m;      // in [0, 2m)
                                r = min(r, r - m);
                                if (accumulate) {
                                    r += __byte_perm(ow[q], 0, 0x4440 + b);
                                    r = min(r, r - m);
                                }
                                r4[b] = r;
                            }
                            w[q] = __byte_perm(__byte_perm(r4[0], r4[1], 0x0040), __byte_perm(r4[2], r4[3], 0x0040), 0x5410);
                        }
                        *reinterpret_cast<uint4*>(blk) = make_uint4(w[0], w[1], w[2], w[3]);
                        *reinterpret_cast<uint4*>(blk + 16) = make_uint4(w[4], w[5], w[6], w[7]);
                    }
                    if (cc + 1 < kChunks) dev::tmem_load_wait();
                }
                dev::tc_fence_before();
                __syncwarp();
                if (lane == 0) dev::mbar_arrive(acc_empty(acc));
            }
            }
            if constexpr (CRTF) {
                // every modulus of the tile is in: reconstruct this lane's column j for the 64 rows
                // i of this warp's half, four entries per word, eight words per pass
                if (ok) {
                    dev::tmem_store_wait();
                    const GemmItem* __restrict__ I = J.I;
                    const int tk = I->crt_tk, s_ = I->s;
                    const int64_t j = static_cast<int64_t>(J.tj) * kGemmJ + quarter * 32 + lane;
                    const int64_t mm = I->m, nn = I->n;
                    const int Ej = j < nn ? exponent_of(I->crt_maxB[j], tk) : 0;
                    const uint32_t rbase = tmem_base + (static_cast<uint32_t>(quarter * 32) << 16) +
                                           static_cast<uint32_t>(2 * BN + 128 * half);
#pragma unroll 1
                    for (int wb = 0; wb < 2; ++wb) {
                        uint32_t R8[kCrtFusedMaxS][8];
#pragma unroll
                        for (int t2 = 0; t2 < kCrtFusedMaxS; ++t2) {
                            if (t2 < s_) {
                                dev::tmem_load_32x8(rbase + 16 * t2 + 8 * wb, R8[t2]);
                            } else {
#pragma unroll
                                for (int q = 0; q < 8; ++q) R8[t2][q] = 0;
                            }
                        }
                        dev::tmem_load_wait();
#pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            uint32_t lo[4], hi[4];  // moduli 0..3 and 4..7 of the word's four entries
                            transpose4(R8[0][q], R8[1][q], R8[2][q], R8[3][q], lo);
                            transpose4(R8[4][q], R8[5][q], R8[6][q], R8[7][q], hi);
#pragma unroll
                            for (int e = 0; e < 4; ++e) {
                                const int64_t i = static_cast<int64_t>(J.ti) * BN + half * 64 + 4 * (8 * wb + q) + e;
                                if (i < mm && j < nn) {
                                    const int De = exponent_of(I->crt_maxA[i], tk);
                                    const bool nonfinite = De == kNonFinite || Ej == kNonFinite;
                                    const uint32_t R[2] = {lo[e], hi[e]};
                                    double v = crt_value<kCrtFusedMaxS, 2>(R, P.cc, nonfinite ? 0 : De + Ej);
                                    if (nonfinite) v = __longlong_as_double(0x7FF8000000000000ll);
                                    double* cp = I->C + i + j * I->ldc;
                                    // the reference's unfused alpha*v + beta*c, one rounding per operation
                                    const double av = __dmul_rn(I->crt_alpha, v);
                                    *cp = I->crt_beta == 0.0 ? av : __dadd_rn(av, __dmul_rn(I->crt_beta, *cp));
                                }
                            }
                        }
                    }
                    dev::tc_fence_before();
                }
            }
        }
        if constexpr (CRTF) dev::tmem_store_wait();  // no residue store in flight when TMEM is freed
    }
    __syncwarp();
    dev::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        dev::tc_fence_after();
        dev::tmem_dealloc(tmem_base, kTmemCols);
    }
}

// failure-path test settings, read at every launch (process-wide)
std::atomic<uint64_t> g_wait_ns{dev::kWaitLimitNs};
std::atomic<int> g_stall{0};

GemmParams make_params(const GemmItem* d_items, int count, int group_j, int64_t jobs, int* err) {
    return GemmParams{d_items, count, group_j, jobs, err, g_wait_ns.load(), g_stall.load()};
}

template <int BN, int KIND = kKindResidue>
void launch_bn(const GemmParams& P, int grid, cudaStream_t st) {
    gemm_i8_modm_kernel<BN, KIND><<<grid, kGemmThreads, Cfg<BN>::kSmemBytes, st>>>(P);
}

}  // namespace

cudaError_t prepare_gemm_kernels() {
    cudaError_t e = cudaFuncSetAttribute(gemm_i8_modm_kernel<256, kKindResidue>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg<256>::kSmemBytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(gemm_i8_modm_kernel<128, kKindResidue>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 Cfg<128>::kSmemBytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(gemm_i8_modm_kernel<256, kKindOz1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 Cfg<256>::kSmemBytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(gemm_i8_modm_kernel<256, kKindCert>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 Cfg<256>::kSmemBytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(gemm_i8_modm_kernel<128, kKindCrt>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 Cfg<128>::kSmemBytes);
    if (e == cudaSuccess) e = prepare_split_kernels();
    if (e == cudaSuccess) e = prepare_crt_kernels();
    return e;
}

void set_gemm_failure_test(uint64_t wait_ns, int stall) {
    g_wait_ns.store(wait_ns ? wait_ns : dev::kWaitLimitNs);
    g_stall.store(stall ? 1 : 0);
}

int64_t gemm_tiles_i(int64_t m, int bn) { return ceil_div(m, bn); }

void launch_gemm(const GemmItem* d_items, int count, int64_t jobs, const GemmConfig& cfg, int num_sms, int* err,
                 cudaStream_t st) {
    if (count <= 0 || jobs <= 0) return;
    const GemmParams P = make_params(d_items, count, cfg.group_j > 0 ? cfg.group_j : 16, jobs, err);
    const int ctas = cfg.ctas > 0 ? std::min(cfg.ctas, num_sms) : num_sms;
    const int grid = static_cast<int>(std::min<int64_t>(ctas, jobs));
    if (cfg.bn == 128) launch_bn<128>(P, grid, st);
    else launch_bn<256>(P, grid, st);
}

void launch_gemm_oz1(const GemmItem* d_items, int count, int64_t jobs, const GemmConfig& cfg, int num_sms, int* err,
                     cudaStream_t st) {
    if (count <= 0 || jobs <= 0) return;
    const GemmParams P = make_params(d_items, count, cfg.group_j > 0 ? cfg.group_j : 16, jobs, err);
    const int grid = static_cast<int>(std::min<int64_t>(num_sms, jobs));
    launch_bn<256, kKindOz1>(P, grid, st);
}

namespace {
std::atomic<int> g_crt_fusion{0};
}  // namespace

void set_crt_fusion(int on) { g_crt_fusion.store(on ? 1 : 0); }
int crt_fusion() { return g_crt_fusion.load(); }

void launch_gemm_crt(const GemmItem* d_items, int count, int64_t jobs, const Plan& plan, int group_j, int num_sms,
                     int* err, cudaStream_t st) {
    if (count <= 0 || jobs <= 0) return;
    GemmParams P = make_params(d_items, count, group_j > 0 ? group_j : 16, jobs, err);
    crt_constants(plan, P.cc);
    const int grid = static_cast<int>(std::min<int64_t>(num_sms, jobs));
    launch_bn<128, kKindCrt>(P, grid, st);
}

void launch_gemm_cert(const GemmItem* d_items, int count, int64_t jobs, int num_sms, int* err, cudaStream_t st) {
    if (count <= 0 || jobs <= 0) return;
    const GemmParams P = make_params(d_items, count, 16, jobs, err);
    const int grid = static_cast<int>(std::min<int64_t>(num_sms, jobs));
    launch_bn<256, kKindCert>(P, grid, st);
}

}  // namespace oz2
