// oz2_crt.cu - CRT reconstruction of the Ozaki-II path: per C entry, s residues r_t in
// [0, m_t) -> the exact integer x = Sum_t r_t W_t - q M (|x| <= M/4, q = rint(Sum_t r_t y_t/m_t)
// from an FP32 estimate) -> one round-to-nearest-even to a double -> * 2^-(D_i + E_j) ->
// alpha/beta update. Ref src/ozaki2_gpu.hpp:526-588 (CrtAcc), :603-626 (launch_crt),
// :628-664 (launch_crt_cplx, 3M recombination Re = P0 - P1, Im = P2 - P0 - P1).
//
// Bandwidth-bound: s bytes of residues per entry in (3s for complex), 8 (16) bytes of C out,
// plus 8 (16) in when beta != 0. Each thread handles 4 consecutive rows of one column.
#include <algorithm>
#include <atomic>
#include <cstring>

#include "oz2_kernels.cuh"
#include "oz2_crt_math.cuh"
#include "oz2_ptx.cuh"

namespace oz2 {
namespace {

struct CrtParams {
    const CrtItem* items;
    int count;
    CrtConst cc;
    uint32_t mod_m[kMaxModuliExt];
};

__device__ __forceinline__ uint32_t sub_mod(uint32_t a, uint32_t b, uint32_t m) {  // (a - b) mod m, a,b < m
    uint32_t r = a + m - b;
    return min(r, r - m);
}

// low bytes of a, b, c, d as one little-endian word
__device__ __forceinline__ uint32_t pack4(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    return __byte_perm(__byte_perm(a, b, 0x0040), __byte_perm(c, d, 0x0040), 0x5410);
}

// Occupancy for the latency-bound loads: real plans of up to 5 limbs (20 moduli) fit 64 registers
// (four blocks per SM), of 6 limbs (21 to 25 moduli) 80 (three); complex ones 128 (two); larger
// real ones take what the reconstruction needs.
template <int S, bool CPLX>
constexpr int crt_min_blocks() { return CPLX ? 2 : (limbs_for(S) <= 5 ? 4 : (limbs_for(S) <= 6 ? 3 : 1)); }
template <int S, bool CPLX>
__global__ void __launch_bounds__(256, crt_min_blocks<S, CPLX>()) crt_kernel(const __grid_constant__ CrtParams P) {
    constexpr int NL = limbs_for(S);
    int lo = 0, hi = P.count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (P.items[mid].block0 <= static_cast<int64_t>(blockIdx.x)) lo = mid;
        else hi = mid - 1;
    }
    const CrtItem* __restrict__ I = P.items + lo;
    const int64_t local = static_cast<int64_t>(blockIdx.x) - I->block0;
    int64_t jblk, ib;
    divmod_index(local, I->iblocks, jblk, ib);
    const int tq = I->tq;
    const int64_t j = jblk * I->jb + threadIdx.x / tq;
    const int64_t i0 = (ib * tq + threadIdx.x % tq) * 4;
    const int64_t m = I->m;
    if (i0 >= m || j >= I->n) return;
    const int tk = I->tk;
    const double ar = I->ar, ai = I->ai, br = I->br, bi = I->bi;
    const int64_t rstride = I->rstride, gstride = I->gstride;
    {
        const int Ej = exponent_of(I->maxB[j], tk);
        const uint8_t* base = I->resid + (i0 >> 5) * (32 * I->n) + j * 32 + (i0 & 31);
        // one 32-bit word per plane = the residues of the 4 entries i0..i0+3
        constexpr int Q = (S + 3) / 4;
        uint32_t w0[4 * Q], w1[CPLX ? 4 * Q : 1], w2[CPLX ? 4 * Q : 1];
#pragma unroll
        for (int t = 0; t < 4 * Q; ++t) {
            w0[t] = t < S ? __ldg(reinterpret_cast<const uint32_t*>(base + t * rstride)) : 0u;
            if (CPLX) {
                w1[t] = t < S ? __ldg(reinterpret_cast<const uint32_t*>(base + gstride + t * rstride)) : 0u;
                w2[t] = t < S ? __ldg(reinterpret_cast<const uint32_t*>(base + 2 * gstride + t * rstride)) : 0u;
            }
        }
        // real: the residue bytes regrouped per entry, four moduli per word
        uint32_t Rq[CPLX ? 1 : 4][CPLX ? 1 : Q];
        if constexpr (!CPLX) {
#pragma unroll
            for (int g = 0; g < Q; ++g) {
                uint32_t o[4];
                transpose4(w0[4 * g], w0[4 * g + 1], w0[4 * g + 2], w0[4 * g + 3], o);
#pragma unroll
                for (int e = 0; e < 4; ++e) Rq[e][g] = o[e];
            }
        }
        // real: the sums of two entries together, each weight read once per pair (four entries'
        // limb sums would cost registers, and so occupancy)
        constexpr int EG = CPLX ? 1 : 2;
        uint32_t ufg[EG];
        uint64_t accg[EG][CPLX ? 1 : NL];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int64_t i = i0 + e;
            if (i >= m) break;
            if constexpr (!CPLX) {
                if (e % EG == 0)
                    crt_sums<S, NL, EG>(*reinterpret_cast<const uint32_t(*)[EG][Q]>(&Rq[e][0]), P.cc, ufg, accg);
            }
            const int De = exponent_of(I->maxA[i], tk);
            const bool nonfinite = De == kNonFinite || Ej == kNonFinite;
            const int shift = nonfinite ? 0 : De + Ej;
            const uint32_t sel = 0x4440 + e;  // byte e of a word, zero-extended
            double* cp = I->C + (CPLX ? 2 : 1) * (i + j * I->ldc);
            if constexpr (!CPLX) {
                double v = crt_finish<NL>(accg[e % EG], static_cast<int64_t>(ufg[e % EG] >> 16), P.cc.M, shift);
                if (nonfinite) v = __longlong_as_double(0x7FF8000000000000ll);
                // the reference's unfused alpha*v + beta*c, one rounding per operation
                const double av = __dmul_rn(ar, v);
                cp[0] = br == 0.0 ? av : __dadd_rn(av, __dmul_rn(br, cp[0]));
            } else {
                uint32_t rr[4 * Q], ri[4 * Q];
#pragma unroll
                for (int t = 0; t < 4 * Q; ++t) {
                    if (t < S) {
                        const uint32_t m = P.mod_m[t];
                        const uint32_t p0 = __byte_perm(w0[t], 0, sel), p1 = __byte_perm(w1[t], 0, sel);
                        const uint32_t p2 = __byte_perm(w2[t], 0, sel);
                        rr[t] = sub_mod(p0, p1, m);                  // Re = P0 - P1
                        ri[t] = sub_mod(sub_mod(p2, p0, m), p1, m);  // Im = P2 - P0 - P1
                    } else {
                        rr[t] = ri[t] = 0;
                    }
                }
                uint32_t Rr[Q], Ri[Q];
#pragma unroll
                for (int g = 0; g < Q; ++g) {
                    Rr[g] = pack4(rr[4 * g], rr[4 * g + 1], rr[4 * g + 2], rr[4 * g + 3]);
                    Ri[g] = pack4(ri[4 * g], ri[4 * g + 1], ri[4 * g + 2], ri[4 * g + 3]);
                }
                double vr = crt_value<S, NL>(Rr, P.cc, shift);
                double vi = crt_value<S, NL>(Ri, P.cc, shift);
                if (nonfinite) vr = vi = __longlong_as_double(0x7FF8000000000000ll);
                double orr = __dsub_rn(__dmul_rn(ar, vr), __dmul_rn(ai, vi));
                double oi = __dadd_rn(__dmul_rn(ar, vi), __dmul_rn(ai, vr));
                if (br != 0.0 || bi != 0.0) {
                    const double cr = cp[0], ci = cp[1];
                    orr = __dadd_rn(orr, __dsub_rn(__dmul_rn(br, cr), __dmul_rn(bi, ci)));
                    oi = __dadd_rn(oi, __dadd_rn(__dmul_rn(br, ci), __dmul_rn(bi, cr)));
                }
                cp[0] = orr;
                cp[1] = oi;
            }
        }
    }
}

// ---------------------------------------------------------------- tensor-core CRT (real)
// The limb sums sum_t r_t W_t are a small integer matrix product: per entry e, D[e][b] = sum_t
// r_et Wb[t][b] with r_et the residue bytes and Wb[t][b] byte b of W_t (b < 4 NL), plus two
// columns of the 16-bit quotient fractions F16_t (low and high byte). One tcgen05.mma kind::i8
// (unsigned bytes, M = 128 entries, N = NC columns, K = 32 moduli, zero-padded) computes them
// for 128 entries; every sum is below 32 * 255^2 < 2^21, exact in the int32 accumulators. The
// threads then do only the byte-to-limb combination, the carry chain and the rounding of the
// dp2a kernel (crt_finish), so the results are the same bits, with 4 NL + 2 TMEM columns read
// per entry in place of 2 Q (2 NL + 1) dp2a.
// A super-tile is 32 rows i x 16 columns j, four MMA tiles g of 32 rows x 4 columns; their
// residues share one 128-byte swizzled A tile (tile g in K bytes 32 g .. 32 g + 31 of each row,
// row 32 c + l = entry (i0 + crt_tc_row(l), j0 + 4 g + c)). 8 warps: for the loads, warp w takes columns w and
// w + 8 of the super-tile; for the epilogue, warp w reads TMEM lane quarter w % 4 of tiles
// w / 4 and w / 4 + 2, so each thread finishes two entries and each warp stores 32 consecutive
// entries of a column. Double-buffered (two A tiles, 2 x 4 NC TMEM columns), persistent, two
// CTAs per SM (NC = 32: 4 NL + 2 <= 32, so NL <= 7) or one (NC = 64, NL = 8).
constexpr int kCrtThreads = 256;
template <int NL>
struct CrtTc {
    static constexpr int NC = 4 * NL + 2 <= 32 ? 32 : 64;  // MMA N and TMEM columns per MMA tile
    static constexpr uint32_t kTmemCols = 2 * 4 * NC;
    static constexpr uint32_t kIdesc = (2u << 4)             // D: s32; A, B: unsigned 8-bit, K-major
                                       | (static_cast<uint32_t>(NC >> 3) << 17) | (static_cast<uint32_t>(128 >> 4) << 24);
    static constexpr int kSmem = 1024 + 2 * 128 * 128 + NC * 128 + 64;  // align slack, two A tiles, B, barriers + slot
    static constexpr int kSmemLaunch = NC == 32 ? 100 * 1024 : 120 * 1024;  // CTAs per SM as TMEM allows
};

struct CrtTcParams {
    const CrtItem* items;
    int count;
    int64_t tiles;  // super-tiles
    int s, nl;
    uint32_t M[kMaxLimbs];
    alignas(16) uint8_t wb[64][32];  // B operand rows: byte b of W_t for t = 0..31 (zero past s); F16 bytes at 4 nl, 4 nl + 1
    int* err;
    uint64_t wait_ns;
};

struct SuperTile {
    const CrtItem* I;
    int64_t i0, j0;
};
// the residue words of super-tile column c (0..15) for this thread: rows i0 + 4 (lane % 8) .. + 3,
// moduli 8 (lane / 8) .. + 7 (one 32-bit word = 4 rows of one modulus; zero past s or n)
__device__ __forceinline__ void crt_tc_load(const SuperTile& T, int c, int s, uint32_t (&wv)[8]) {
    const int lane = threadIdx.x & 31;
    const int64_t j = T.j0 + c, n = T.I->n;
    const int rq = lane & 7, mg = lane >> 3;
    const uint8_t* base = T.I->resid + (T.i0 >> 5) * (32 * n) + j * 32 + 4 * rq;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const int t = 8 * mg + u;
        wv[u] = j < n && t < s ? __ldg(reinterpret_cast<const uint32_t*>(base + t * T.I->rstride)) : 0u;
    }
}
// Entry rows within a 32-row group are permuted in the A tile (and so in the TMEM lanes): row
// l = 4 a + u sits in lane a + 8 u, so the eight row quads of one store instruction land in eight
// different swizzle phases (no bank conflicts); lane -> row is crt_tc_row.
__device__ __forceinline__ int crt_tc_row(int lane) { return 4 * (lane & 7) + (lane >> 3); }
// the words of column c regrouped per entry (4 x 4 byte transposes): 8 bytes per entry into row
// 32 (c % 4) + (lane % 8) + 8 u of the A tile, K bytes 32 (c / 4) + 8 (lane / 8) .. + 7
__device__ __forceinline__ void crt_tc_store(uint8_t* sA, int c, const uint32_t (&wv)[8]) {
    const int lane = threadIdx.x & 31;
    const int rq = lane & 7, mg = lane >> 3, g = c >> 2;
    uint32_t lo[4], hi[4];
    transpose4(wv[0], wv[1], wv[2], wv[3], lo);
    transpose4(wv[4], wv[5], wv[6], wv[7], hi);
    const int chunk = 2 * g + (mg >> 1);  // 16-byte chunk of the row's 128 K bytes
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int e = 32 * (c & 3) + rq + 8 * u;  // entry row 4 rq + u of the group
        *reinterpret_cast<uint2*>(sA + e * 128 + ((chunk ^ (e & 7)) << 4) + 8 * (mg & 1)) = make_uint2(lo[u], hi[u]);
    }
}

// The row and column maxima this thread needs to finish its two entries of a super-tile: row
// i0 + crt_tc_row(lane), columns j0 + 4 (warp / 4) + warp % 4 and 8 further (zero outside the
// problem). Loaded with the super-tile's residues, a loop iteration before they are used, so
// finishing waits on no global load.
struct TcMaxima {
    unsigned long long a, b0, b1;
};
__device__ __forceinline__ TcMaxima crt_tc_maxima(const SuperTile& T) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t i = T.i0 + crt_tc_row(lane);
    const int64_t j0 = T.j0 + 4 * (warp >> 2) + (warp & 3), j1 = j0 + 8;
    TcMaxima r;
    r.a = i < T.I->m ? __ldg(T.I->maxA + i) : 0ull;
    r.b0 = j0 < T.I->n ? __ldg(T.I->maxB + j0) : 0ull;
    r.b1 = j1 < T.I->n ? __ldg(T.I->maxB + j1) : 0ull;
    return r;
}

// Software-pipelined over the CTA's super-tiles: while the MMAs of super-tile k run, the threads
// load super-tile k + 1's residues into registers and finish super-tile k - 1 from the other
// accumulators.
template <int NL>
__global__ void __launch_bounds__(kCrtThreads) crt_tc_kernel(const __grid_constant__ CrtTcParams P) {
    using T = CrtTc<NL>;
    constexpr int NC = T::NC;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t{1023});
    uint8_t* sA0 = smem;                 // two 128 rows x 128 B tiles, K-major, 128-byte swizzle
    uint8_t* sB = smem + 2 * 128 * 128;  // NC rows x 128 B
    uint64_t* bar = reinterpret_cast<uint64_t*>(sB + NC * 128);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 2);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x < NC) {  // B: the W bytes of the plan (only the 32 K bytes of each row are read)
        const int b = threadIdx.x;
        const uint4* src = reinterpret_cast<const uint4*>(P.wb[b]);
#pragma unroll
        for (int c = 0; c < 2; ++c) *reinterpret_cast<uint4*>(sB + b * 128 + ((c ^ (b & 7)) << 4)) = src[c];
    }
    if (threadIdx.x == 0) {
        dev::mbar_init(dev::smem_addr(bar), 1);
        dev::mbar_init(dev::smem_addr(bar + 1), 1);
        *abort_flag = 0;
        dev::fence_barrier_init();
    }
    if (warp == 0) {
        dev::tmem_alloc(dev::smem_addr(tmem_slot), T::kTmemCols);
        dev::tmem_relinquish();
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    dev::tc_fence_before();
    __syncthreads();
    dev::tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    int item = 0;
    {  // the item of this CTA's first super-tile; later ones only move forward
        int hi = P.count - 1;
        while (item < hi) {
            const int mid = (item + hi + 1) >> 1;
            if (P.items[mid].block0 <= static_cast<int64_t>(blockIdx.x)) item = mid;
            else hi = mid - 1;
        }
    }
    auto tile_ref = [&](int64_t tile) {
        while (item + 1 < P.count && P.items[item + 1].block0 <= tile) ++item;
        const CrtItem* I = P.items + item;
        const int64_t local = tile - I->block0;
        int64_t qd, rm;
        divmod_index(local, I->iblocks, qd, rm);
        return SuperTile{I, rm * 32, qd * 16};
    };
    const int64_t ntiles = P.tiles > blockIdx.x ? (P.tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    uint32_t wv[2][8];
    SuperTile cur{}, prev{};
    TcMaxima mcur{}, mprev{};
    if (ntiles > 0) {
        cur = tile_ref(blockIdx.x);
        crt_tc_load(cur, warp, P.s, wv[0]);
        crt_tc_load(cur, warp + 8, P.s, wv[1]);
        mcur = crt_tc_maxima(cur);
    }
    bool ok = true;
    uint32_t committed = 0, last_par = 0;  // (thread 0) per accumulator: a commit issued, its parity
    for (int64_t kk = 0; kk <= ntiles && ok; ++kk) {
        const int buf = static_cast<int>(kk & 1);
        if (kk < ntiles) {
            crt_tc_store(sA0 + buf * 128 * 128, warp, wv[0]);
            crt_tc_store(sA0 + buf * 128 * 128, warp + 8, wv[1]);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        }
        dev::tc_fence_before();
        __syncthreads();
        if (kk < ntiles && threadIdx.x == 0) {
            dev::tc_fence_after();
            const uint32_t a0 = dev::smem_addr(sA0 + buf * 128 * 128);
#pragma unroll
            for (int g = 0; g < 4; ++g)
                dev::mma_i8(tmem + static_cast<uint32_t>((4 * buf + g) * NC), dev::sw128_kmajor_desc(a0 + 32 * g),
                            dev::sw128_kmajor_desc(dev::smem_addr(sB)), T::kIdesc, 0u);
            dev::tc_commit(dev::smem_addr(bar + buf));
            committed |= 1u << buf;
            last_par = (last_par & ~(1u << buf)) | (static_cast<uint32_t>((kk >> 1) & 1) << buf);
        }
        SuperTile nxt{};
        TcMaxima mnxt{};
        if (kk + 1 < ntiles) {  // the next super-tile's loads run under this iteration's waits and arithmetic
            nxt = tile_ref(blockIdx.x + (kk + 1) * gridDim.x);
            crt_tc_load(nxt, warp, P.s, wv[0]);
            crt_tc_load(nxt, warp + 8, P.s, wv[1]);
            mnxt = crt_tc_maxima(nxt);
        }
        if (kk > 0) {  // finish super-tile kk - 1
            const int pb = buf ^ 1;
            const uint32_t parity = static_cast<uint32_t>(((kk - 1) >> 1) & 1);
            int w_ok = 1;  // one thread waits; the others sleep in the block barrier
            if (threadIdx.x == 0)
                w_ok = dev::mbar_wait(dev::smem_addr(bar + pb), parity, abort_flag, P.err, dev::kErrTimeoutAccFull,
                                      P.wait_ns) ? 1 : 0;
            if (!__syncthreads_and(w_ok)) {
                ok = false;
                break;
            }
            dev::tc_fence_after();
            const CrtItem* __restrict__ I = prev.I;
            const int q = warp & 3, h = warp >> 2;
            const int64_t i = prev.i0 + crt_tc_row(lane);
            const int tk = I->tk;
            const int De = i < I->m ? exponent_of(mprev.a, tk) : 0;
#pragma unroll
            for (int gg = 0; gg < 2; ++gg) {
                const int g = h + 2 * gg;
                uint32_t d[NC];
                const uint32_t taddr = tmem + (static_cast<uint32_t>(32 * q) << 16) + static_cast<uint32_t>((4 * pb + g) * NC);
                dev::tmem_load_32x32(taddr, *reinterpret_cast<uint32_t(*)[32]>(d));
                if constexpr (NC == 64) dev::tmem_load_32x32(taddr + 32, *reinterpret_cast<uint32_t(*)[32]>(d + 32));
                dev::tmem_load_wait();
                const int64_t j = prev.j0 + 4 * g + q;
                if (i < I->m && j < I->n) {
                    uint64_t acc[NL];
#pragma unroll
                    for (int l = 0; l < NL; ++l) {
                        const uint32_t lo = d[4 * l] + (d[4 * l + 1] << 8);      // < 2^30
                        const uint32_t hi = d[4 * l + 2] + (d[4 * l + 3] << 8);  // < 2^30
                        acc[l] = static_cast<uint64_t>(lo) + (static_cast<uint64_t>(hi) << 16);
                    }
                    const uint32_t uf = (1u << 15) + d[4 * NL] + (d[4 * NL + 1] << 8);
                    const int64_t qv = static_cast<int64_t>(uf >> 16);
                    const int Ej = exponent_of(gg ? mprev.b1 : mprev.b0, tk);
                    const bool nonfinite = De == kNonFinite || Ej == kNonFinite;
                    double v = crt_finish<NL>(acc, qv, P.M, nonfinite ? 0 : De + Ej);
                    if (nonfinite) v = __longlong_as_double(0x7FF8000000000000ll);
                    double* cp = I->C + i + j * I->ldc;
                    // the reference's unfused alpha*v + beta*c, one rounding per operation
                    const double av = __dmul_rn(I->ar, v);
                    *cp = I->br == 0.0 ? av : __dadd_rn(av, __dmul_rn(I->br, *cp));
                }
            }
        }
        prev = cur;
        cur = nxt;
        mprev = mcur;
        mcur = mnxt;
    }
    if (!ok && threadIdx.x == 0) {  // the last MMA of each accumulator completes before TMEM is freed
        for (int b = 0; b < 2; ++b)
            if (committed & (1u << b)) dev::mbar_wait_drain(dev::smem_addr(bar + b), (last_par >> b) & 1u);
    }
    dev::tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        dev::tc_fence_after();
        dev::tmem_dealloc(tmem, T::kTmemCols);
    }
}

// complex CRTs stop at s = 24 (zgemm is the reference's call); the extended sets are real only
template <int S>
void crt_launch_s(const CrtParams& P, int64_t blocks, bool cplx, cudaStream_t st) {
    if constexpr (S <= kMaxModuli) {
        if (cplx) {
            crt_kernel<S, true><<<static_cast<unsigned>(blocks), 256, 0, st>>>(P);
            return;
        }
    }
    crt_kernel<S, false><<<static_cast<unsigned>(blocks), 256, 0, st>>>(P);
}

template <int S>
void crt_dispatch(int s, const CrtParams& P, int64_t blocks, bool cplx, cudaStream_t st) {
    if constexpr (S <= kMaxModuliExt) {
        if (s == S) return crt_launch_s<S>(P, blocks, cplx, st);
        crt_dispatch<S + 1>(s, P, blocks, cplx, st);
    }
}

// the parameter block is copied with every launch: size classes keep small blobs cheap
template <int N>
struct alignas(16) BlobParam {
    unsigned char data[N];
    uint32_t bytes;
};
template <int N>
__global__ void write_blob_kernel(const __grid_constant__ BlobParam<N> b, unsigned char* dst) {
    for (uint32_t i = threadIdx.x * 16; i < b.bytes; i += blockDim.x * 16)
        *reinterpret_cast<uint4*>(dst + i) = *reinterpret_cast<const uint4*>(b.data + i);
}
template <int N>
void write_blob_n(const unsigned char* src, size_t n, unsigned char* dst, cudaStream_t st) {
    static thread_local BlobParam<N> bp;
    std::memcpy(bp.data, src, n);
    bp.bytes = static_cast<uint32_t>((n + 15) & ~size_t{15});
    write_blob_kernel<N><<<1, 256, 0, st>>>(bp, dst);
}

// VEC: both pointers 16-byte aligned, 16-byte words first
template <bool VEC>
__global__ void sm_copy_kernel(const unsigned char* __restrict__ src, unsigned char* __restrict__ dst, size_t bytes) {
    const size_t tid = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    size_t tail = 0;
    if (VEC) {
        const size_t n16 = bytes / 16;
        for (size_t i = tid; i < n16; i += stride)
            reinterpret_cast<uint4*>(dst)[i] = reinterpret_cast<const uint4*>(src)[i];
        tail = n16 * 16;
    }
    for (size_t i = tail + tid; i < bytes; i += stride) dst[i] = src[i];
}

template <bool VEC>
__global__ void fill_kernel(unsigned char* __restrict__ dst, uint32_t word, size_t bytes) {
    const size_t tid = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    size_t tail = 0;
    if (VEC) {
        const size_t n16 = bytes / 16;
        for (size_t i = tid; i < n16; i += stride) reinterpret_cast<uint4*>(dst)[i] = make_uint4(word, word, word, word);
        tail = n16 * 16;
    }
    for (size_t i = tail + tid; i < bytes; i += stride) dst[i] = static_cast<unsigned char>(word);
}

// blocks of 256 threads for `units` units of work, at most 4 per SM of a B200
unsigned copy_blocks(size_t units) {
    return static_cast<unsigned>(std::min<size_t>((units + 255) / 256 + 1, 4 * 148));
}

__global__ void scale_c_kernel(double* C, int64_t ldc, int64_t m, int64_t n, double br, double bi, int cplx) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= m) return;
    for (int64_t j = blockIdx.y; j < n; j += gridDim.y) {
        if (!cplx) {
            double* cp = C + i + j * ldc;
            *cp = br == 0.0 ? 0.0 : __dmul_rn(br, *cp);
        } else {
            double* cp = C + 2 * (i + j * ldc);
            if (br == 0.0 && bi == 0.0) {
                cp[0] = 0.0;
                cp[1] = 0.0;
            } else {
                const double r = cp[0], im = cp[1];
                cp[0] = __dsub_rn(__dmul_rn(br, r), __dmul_rn(bi, im));
                cp[1] = __dadd_rn(__dmul_rn(br, im), __dmul_rn(bi, r));
            }
        }
    }
}

// Ozaki Scheme I (the reference's comparison baseline, benchmarks/ozaki1_gpu.hpp:50-75): the
// exact diagonal sums S_d, most significant first, in double-double Horner steps T = 128 T + S_d
// (scaling by 128 is exact, so a contracted multiply-add rounds as the separate operations do),
// then one ldexp by 7 (L - 1) - D_i - E_j, NaN for non-finite rows / columns. The sums are
// stored row-major (acc[d][i n + j]); a block takes a 32 x 32 tile, reads it along j and writes
// C along i through shared memory. Block (32, 8), grid (ceil(n / 32), rows of tiles strided).
__global__ void __launch_bounds__(256) oz1_horner_kernel(const int64_t* __restrict__ acc, int64_t m, int64_t n, int L,
                                                         const unsigned long long* __restrict__ maxA,
                                                         const unsigned long long* __restrict__ maxB, int tk,
                                                         double* __restrict__ C, int64_t ldc) {
    __shared__ double tile[32][33];
    const int64_t j0 = static_cast<int64_t>(blockIdx.x) * 32, plane = m * n;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int64_t j = j0 + tx;
    const int Ej = j < n ? exponent_of(maxB[j], tk) : 0;
    for (int64_t i0 = static_cast<int64_t>(blockIdx.y) * 32; i0 < m; i0 += static_cast<int64_t>(gridDim.y) * 32) {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int64_t i = i0 + ty + 8 * r;
            if (i >= m || j >= n) continue;
            const int Di = exponent_of(maxA[i], tk);
            double hi = 0.0, lo = 0.0;
            for (int d = 0; d < L; ++d) {
                const double sd = static_cast<double>(acc[d * plane + i * n + j]);
                if (d > 0) {
                    hi *= 128.0;
                    lo *= 128.0;
                }
                const double sm = hi + sd, bb = sm - hi;
                const double err = (hi - (sm - bb)) + (sd - bb) + lo;
                hi = sm + err;
                lo = err - (hi - sm);
            }
            double v = ldexp(hi + lo, 7 * (L - 1) - Di - Ej);
            if (Di == kNonFinite || Ej == kNonFinite) v = __longlong_as_double(0x7FF8000000000000ll);
            tile[ty + 8 * r][tx] = v;
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int64_t jj = j0 + ty + 8 * r, ii = i0 + tx;
            if (ii < m && jj < n) C[ii + jj * ldc] = tile[tx][ty + 8 * r];
        }
        __syncthreads();
    }
}

}  // namespace

int64_t crt_item_blocks(CrtItem& it, int64_t block0) {
    it.block0 = block0;
    if (it.mma) {  // tensor-core CRT: super-tiles of 32 rows x 16 columns
        it.iblocks = ceil_div(it.m, 32);
        return it.m > 0 ? it.iblocks * ceil_div(it.n, 16) : 0;
    }
    const int64_t quads = ceil_div(it.m, 4);
    int tq = 1;
    while (tq < 8 && tq < quads) tq *= 2;  // a warp reads 4 columns x 32 rows: one 128-byte line per plane
    it.tq = tq;
    it.jb = 256 / tq;
    it.iblocks = ceil_div(quads, tq);
    return it.m > 0 ? ceil_div(it.n, it.jb) * it.iblocks : 0;
}

namespace {
int sm_count() {
    static int cached[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cached[dev]) {
        int v = 0;
        cached[dev] = cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0 ? v : 148;
    }
    return cached[dev];
}

std::atomic<int> g_crt_path{2};

template <int NL>
void crt_tc_launch(const CrtTcParams& P, int64_t blocks, cudaStream_t st) {
    using T = CrtTc<NL>;
    const int per_sm = 512 / static_cast<int>(T::kTmemCols);
    const int grid = static_cast<int>(std::min<int64_t>(blocks, static_cast<int64_t>(sm_count()) * per_sm));
    crt_tc_kernel<NL><<<grid, kCrtThreads, T::kSmemLaunch, st>>>(P);
}

}  // namespace

void set_crt_path(int path) { g_crt_path.store(path); }
int crt_path() { return g_crt_path.load(); }

bool crt_uses_mma(const Plan& plan, bool cplx) {
    const int path = g_crt_path.load();
    return !cplx && (path == 1 || (path == 2 && plan.nl >= kCrtTcMinLimbs));
}

cudaError_t prepare_crt_kernels() {
    cudaError_t e = cudaSuccess;
    auto set = [&](const void* f, int bytes) {
        if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    };
    set(reinterpret_cast<const void*>(crt_tc_kernel<2>), CrtTc<2>::kSmemLaunch);
    set(reinterpret_cast<const void*>(crt_tc_kernel<3>), CrtTc<3>::kSmemLaunch);
    set(reinterpret_cast<const void*>(crt_tc_kernel<4>), CrtTc<4>::kSmemLaunch);
    set(reinterpret_cast<const void*>(crt_tc_kernel<5>), CrtTc<5>::kSmemLaunch);
    set(reinterpret_cast<const void*>(crt_tc_kernel<6>), CrtTc<6>::kSmemLaunch);
    set(reinterpret_cast<const void*>(crt_tc_kernel<7>), CrtTc<7>::kSmemLaunch);
    set(reinterpret_cast<const void*>(crt_tc_kernel<8>), CrtTc<8>::kSmemLaunch);
    return e;
}

void launch_crt(const CrtItem* d_items, int count, int64_t blocks, const Plan& plan, bool cplx, int* err,
                cudaStream_t st) {
    if (crt_uses_mma(plan, cplx)) {
        if (count <= 0 || blocks <= 0) return;
        static thread_local CrtTcParams P;
        P = CrtTcParams{};
        P.items = d_items;
        P.count = count;
        P.tiles = blocks;
        P.s = plan.s;
        P.nl = plan.nl;
        for (int l = 0; l < plan.nl; ++l) P.M[l] = plan.M[l];
        for (int t = 0; t < plan.s; ++t) {
            for (int b = 0; b < 4 * plan.nl; ++b) P.wb[b][t] = static_cast<uint8_t>(plan.W[t][b / 4] >> (8 * (b % 4)));
            // the 16-bit quotient fraction of crt_constants, as two bytes
            const uint64_t f = ((static_cast<uint64_t>(plan.y[t]) << 16) + plan.m[t] / 2) / plan.m[t];
            const uint32_t f16 = static_cast<uint32_t>(std::min<uint64_t>(f, 0xFFFFu));
            P.wb[4 * plan.nl][t] = static_cast<uint8_t>(f16);
            P.wb[4 * plan.nl + 1][t] = static_cast<uint8_t>(f16 >> 8);
        }
        P.err = err;
        P.wait_ns = dev::kWaitLimitNs;
        switch (plan.nl) {
            case 2: crt_tc_launch<2>(P, blocks, st); break;
            case 3: crt_tc_launch<3>(P, blocks, st); break;
            case 4: crt_tc_launch<4>(P, blocks, st); break;
            case 5: crt_tc_launch<5>(P, blocks, st); break;
            case 6: crt_tc_launch<6>(P, blocks, st); break;
            case 7: crt_tc_launch<7>(P, blocks, st); break;
            default: crt_tc_launch<8>(P, blocks, st); break;
        }
        return;
    }
    if (count <= 0 || blocks <= 0) return;
    CrtParams P{};
    P.items = d_items;
    P.count = count;
    crt_constants(plan, P.cc);
    for (int t = 0; t < plan.s; ++t) P.mod_m[t] = plan.m[t];
    crt_dispatch<2>(plan.s, P, blocks, cplx, st);
}

void launch_oz1_horner(const int64_t* acc, int64_t m, int64_t n, int L, const unsigned long long* maxA,
                       const unsigned long long* maxB, int tk, double* C, int64_t ldc, cudaStream_t st) {
    if (m <= 0 || n <= 0) return;
    dim3 grid(static_cast<unsigned>(ceil_div(n, 32)), static_cast<unsigned>(std::min<int64_t>(ceil_div(m, 32), 65535)));
    oz1_horner_kernel<<<grid, dim3(32, 8), 0, st>>>(acc, m, n, L, maxA, maxB, tk, C, ldc);
}

void launch_write_blob(const void* src, size_t bytes, void* dst, cudaStream_t st) {
    const unsigned char* p = static_cast<const unsigned char*>(src);
    for (size_t off = 0; off < bytes; off += kParamBlobBytes) {
        const size_t n = std::min(kParamBlobBytes, bytes - off);
        unsigned char* d = static_cast<unsigned char*>(dst) + off;
        if (n <= 1024) write_blob_n<1024>(p + off, n, d, st);
        else if (n <= 4096) write_blob_n<4096>(p + off, n, d, st);
        else if (n <= 12288) write_blob_n<12288>(p + off, n, d, st);
        else write_blob_n<kParamBlobBytes>(p + off, n, d, st);
    }
}

void launch_sm_copy(const void* src, void* dst, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return;
    const auto* s = static_cast<const unsigned char*>(src);
    auto* d = static_cast<unsigned char*>(dst);
    if (((reinterpret_cast<uintptr_t>(s) | reinterpret_cast<uintptr_t>(d)) & 15) == 0)
        sm_copy_kernel<true><<<copy_blocks(bytes / 16), 256, 0, st>>>(s, d, bytes);
    else
        sm_copy_kernel<false><<<copy_blocks(bytes), 256, 0, st>>>(s, d, bytes);
}

void launch_fill(void* dst, unsigned char value, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return;
    auto* d = static_cast<unsigned char*>(dst);
    const uint32_t word = value * 0x01010101u;
    if ((reinterpret_cast<uintptr_t>(d) & 15) == 0) fill_kernel<true><<<copy_blocks(bytes / 16), 256, 0, st>>>(d, word, bytes);
    else fill_kernel<false><<<copy_blocks(bytes), 256, 0, st>>>(d, word, bytes);
}

void launch_scale_c(double* C, int64_t ldc, int64_t m, int64_t n, const double* beta, bool cplx, cudaStream_t st) {
    if (m <= 0 || n <= 0) return;
    dim3 grid(static_cast<unsigned>(ceil_div(m, 256)), static_cast<unsigned>(std::min<int64_t>(n, 65535)));
    scale_c_kernel<<<grid, 256, 0, st>>>(C, ldc, m, n, beta[0], cplx ? beta[1] : 0.0, cplx ? 1 : 0);
}

}  // namespace oz2
