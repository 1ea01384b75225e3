// oz2_crt.cu - CRT reconstruction of the Ozaki-II path: per C entry, s residues r_t in
// [0, m_t) -> the exact integer x = Sum_t r_t W_t - q M (|x| <= M/4, q = rint(Sum_t r_t y_t/m_t)
// from an FP32 estimate) -> one round-to-nearest-even to a double -> * 2^-(D_i + E_j) ->
// alpha/beta update. Ref src/ozaki2_gpu.hpp:526-588 (CrtAcc), :603-626 (launch_crt),
// :628-664 (launch_crt_cplx, 3M recombination Re = P0 - P1, Im = P2 - P0 - P1).
//
// Bandwidth-bound: s bytes of residues per entry in (3s for complex), 8 (16) bytes of C out,
// plus 8 (16) in when beta != 0. Each thread handles 4 consecutive rows of one column.
#include <algorithm>
#include <cstring>

#include "oz2_kernels.cuh"
#include "oz2_ptx.cuh"

namespace oz2 {
namespace {

struct CrtParams {
    const CrtItem* items;
    int count;
    CrtConst cc;
    uint32_t mod_m[kMaxModuliExt];
};

__device__ __forceinline__ int exponent_of(unsigned long long b, int tk) {
    if (b >= 0x7FF0000000000000ull) return kNonFinite;
    if (b == 0) return 0;
    const int be = static_cast<int>(b >> 52);
    const int e2 = be ? be - 1022 : -1010 - __clzll(static_cast<long long>(b));
    return tk - e2;
}

// 2^E * d for d in [2^63, 2^64]: exponent arithmetic on the bits while the result stays normal
// (exact), ldexp otherwise (overflow, or one rounding into the subnormal range)
__device__ __forceinline__ double scale_pow2(double d, int E) {
    if (E >= -1022 - 63 && E <= 1023 - 64)
        return __longlong_as_double(__double_as_longlong(d) + (static_cast<long long>(E) << 52));
    return ldexp(d, E);
}

// Exact reconstruction + single rounding. R[g] holds the residues r_t in [0, m_t) of the moduli
// 4g..4g+3 as bytes (zero past s). Every sum is a chain of two-way byte dot products (dp2a):
// q = round(Sum r_t y_t / m_t) from the 16-bit fractions F16_t (error below 24 * 255 * 2^-16 <
// 0.1, inside the 1/4 margin that |x| <= M/4 leaves, so q is the reference's FP32 quotient),
// and Sum r_t W_t limb by limb over 16-bit limbs of W_t (each limb sum below 24 * 255 * 2^16 <
// 2^29), then x = Sum r_t W_t - q M modulo 2^(32 NL) in 64-bit words, rounded once to double.
template <int NL>
__device__ __forceinline__ double crt_finish(const uint64_t (&acc)[NL], int64_t q, const uint32_t* Mw, int shift);

template <int S, int NL>
__device__ __forceinline__ double crt_value(const uint32_t (&R)[(S + 3) / 4], const CrtConst& cc, int shift) {
    constexpr int Q = (S + 3) / 4;
    uint32_t uf = 1u << 15;  // rounding offset of the quotient
#pragma unroll
    for (int g = 0; g < Q; ++g) {
        uf = __dp2a_lo(cc.Fq[g][0], R[g], uf);
        uf = __dp2a_hi(cc.Fq[g][1], R[g], uf);
    }
    const int64_t q = static_cast<int64_t>(uf >> 16);
    uint64_t acc[NL];
#pragma unroll
    for (int l = 0; l < NL; ++l) {
        uint32_t a0 = 0, a1 = 0;  // 16-bit limbs 2l and 2l + 1
#pragma unroll
        for (int g = 0; g < Q; ++g) {
            a0 = __dp2a_lo(cc.Wq[g][2 * l][0], R[g], a0);
            a0 = __dp2a_hi(cc.Wq[g][2 * l][1], R[g], a0);
            a1 = __dp2a_lo(cc.Wq[g][2 * l + 1][0], R[g], a1);
            a1 = __dp2a_hi(cc.Wq[g][2 * l + 1][1], R[g], a1);
        }
        acc[l] = static_cast<uint64_t>(a0) + (static_cast<uint64_t>(a1) << 16);
    }
    return crt_finish<NL>(acc, q, cc.M, shift);
}

// From the 32-bit limb sums acc[l] = sum_t r_t W_t[l] (below 2^46) and the quotient q: x = sum_t
// r_t W_t - q M modulo 2^(32 NL) in 64-bit words (|x| <= M/4, two's complement), its magnitude's
// leading 64 bits with a sticky bit for the rest, one RNE to double, 2^-shift.
template <int NL>
__device__ __forceinline__ double crt_finish(const uint64_t (&acc)[NL], int64_t q, const uint32_t* Mw, int shift) {
    uint32_t w[NL];
    int64_t carry = 0;
#pragma unroll
    for (int l = 0; l < NL; ++l) {
        const int64_t v = static_cast<int64_t>(acc[l]) - q * static_cast<int64_t>(Mw[l]) + carry;
        w[l] = static_cast<uint32_t>(v);
        carry = v >> 32;
    }
    // 64-bit words, two's complement -> sign and magnitude
    constexpr int NW = (NL + 1) / 2;
    uint64_t X[NW];
#pragma unroll
    for (int i = 0; i < NW; ++i)
        X[i] = static_cast<uint64_t>(w[2 * i]) | (2 * i + 1 < NL ? static_cast<uint64_t>(w[2 * i + 1]) << 32 : 0);
    if (NL % 2)  // odd word count: sign-extend the top word into the last 64-bit word
        X[NW - 1] = static_cast<uint64_t>(static_cast<int64_t>(static_cast<int32_t>(w[NL - 1])));
    const bool neg = static_cast<int64_t>(X[NW - 1]) < 0;
    if (neg) {
        uint64_t borrow = 1;
#pragma unroll
        for (int i = 0; i < NW; ++i) {
            const uint64_t nv = ~X[i] + borrow;
            borrow = (borrow && nv == 0) ? 1 : 0;
            X[i] = nv;
        }
    }
    // leading 64 bits with a sticky bit for everything below
    uint64_t hiw = 0, low = 0;
    bool sticky = false;
    int tw = -1;
#pragma unroll
    for (int i = NW - 1; i >= 0; --i)
        if (tw < 0 && X[i]) tw = i;
    if (tw < 0) return 0.0;
#pragma unroll
    for (int i = 0; i < NW; ++i) {
        if (i == tw) hiw = X[i];
        else if (i == tw - 1) low = X[i];
        else if (i < tw - 1) sticky |= X[i] != 0;
    }
    const int z = __clzll(static_cast<long long>(hiw));
    const uint64_t top = z ? (hiw << z) | (low >> (64 - z)) : hiw;
    sticky |= (z ? (low << z) : low) != 0;
    const double val = scale_pow2(__ull2double_rn(top | (sticky ? 1u : 0u)), 64 * tw - z - shift);
    return neg ? -val : val;
}

__device__ __forceinline__ uint32_t sub_mod(uint32_t a, uint32_t b, uint32_t m) {  // (a - b) mod m, a,b < m
    uint32_t r = a + m - b;
    return min(r, r - m);
}

// low bytes of a, b, c, d as one little-endian word
__device__ __forceinline__ uint32_t pack4(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    return __byte_perm(__byte_perm(a, b, 0x0040), __byte_perm(c, d, 0x0040), 0x5410);
}

// 4 x 4 byte transpose: word t of `in` holds entries e = 0..3 of modulus 4g + t; word e of `out`
// holds moduli 4g..4g+3 of entry e
__device__ __forceinline__ void transpose4(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t (&out)[4]) {
    const uint32_t t0 = __byte_perm(a, b, 0x5140), t1 = __byte_perm(a, b, 0x7362);
    const uint32_t t2 = __byte_perm(c, d, 0x5140), t3 = __byte_perm(c, d, 0x7362);
    out[0] = __byte_perm(t0, t2, 0x5410);
    out[1] = __byte_perm(t0, t2, 0x7632);
    out[2] = __byte_perm(t1, t3, 0x5410);
    out[3] = __byte_perm(t1, t3, 0x7632);
}

template <int S, bool CPLX>
__global__ void __launch_bounds__(256) crt_kernel(const __grid_constant__ CrtParams P) {
    constexpr int NL = limbs_for(S);
    int lo = 0, hi = P.count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (P.items[mid].block0 <= static_cast<int64_t>(blockIdx.x)) lo = mid;
        else hi = mid - 1;
    }
    const CrtItem* __restrict__ I = P.items + lo;
    const int64_t local = static_cast<int64_t>(blockIdx.x) - I->block0;
    const int64_t jblk = local / I->iblocks, ib = local - jblk * I->iblocks;
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
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int64_t i = i0 + e;
            if (i >= m) break;
            const int De = exponent_of(I->maxA[i], tk);
            const bool nonfinite = De == kNonFinite || Ej == kNonFinite;
            const int shift = nonfinite ? 0 : De + Ej;
            const uint32_t sel = 0x4440 + e;  // byte e of a word, zero-extended
            double* cp = I->C + (CPLX ? 2 : 1) * (i + j * I->ldc);
            if constexpr (!CPLX) {
                double v = crt_value<S, NL>(Rq[e], P.cc, shift);
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

// ---------------------------------------------------------------- tensor-core CRT (real, 8 limbs)
// The limb sums sum_t r_t W_t are a small integer matrix product: per entry e, D[e][b] = sum_t
// r_et Wb[t][b] with r_et the residue bytes and Wb[t][b] byte b of W_t (b < 4 NL), plus two
// columns of the 16-bit quotient fractions F16_t (low and high byte). One tcgen05.mma kind::i8
// (unsigned bytes, M = 128 entries, N = 64 columns, K = 32 moduli, zero-padded) computes them
// for 128 entries: every sum is below 32 * 255^2 < 2^21, exact in the int32 accumulators. The
// threads then do only the carry chain and the rounding of the dp2a kernel (crt_finish), so the
// results are the same bits; the integer-multiply pipe, which bounds the dp2a kernel, is left
// to the few 64-bit products of the carry chain.
// A CTA is 4 warps; a tile is 32 rows i x 4 columns j (warp q: column j0 + q, its lanes the
// rows: TMEM lane 32 q + l is entry (i0 + l, j0 + q), so each warp stores 32 consecutive C
// entries of a column). Persistent over the tiles of all items of the launch.
constexpr int kCrtN = 64;                               // MMA N: 4 NL limb bytes + 2 quotient bytes
constexpr uint32_t kCrtIdesc = (2u << 4)                  // D: s32; A, B: unsigned 8-bit, K-major
                               | (static_cast<uint32_t>(kCrtN >> 3) << 17) | (static_cast<uint32_t>(128 >> 4) << 24);
constexpr int kCrtSmem = 1024 + 2 * 128 * 128 + kCrtN * 128 + 64;  // align slack, two A tiles, B, barriers + slot

struct CrtMmaParams {
    const CrtItem* items;
    int count;
    int64_t tiles;
    int s, nl;
    uint32_t M[kMaxLimbs];
    alignas(16) uint8_t wb[kCrtN][32];  // B operand rows: byte b of W_t for t = 0..31 (zero past s); F16 bytes at 4 nl, 4 nl + 1
    int* err;
    uint64_t wait_ns;
};

// the residue words of one tile for this thread: column j0 + warp, rows i0 + 4 (lane % 8) .. + 3,
// moduli 8 (lane / 8) .. + 7 (one 32-bit word = 4 rows per modulus; zero past s or n)
struct TileRef {
    const CrtItem* I;
    int64_t i0, j0;
};
__device__ __forceinline__ void crt_tile_load(const TileRef& T, int s, uint32_t (&wv)[8]) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t j = T.j0 + warp, n = T.I->n;
    const int rq = lane & 7, mg = lane >> 3;
    const uint8_t* base = T.I->resid + (T.i0 >> 5) * (32 * n) + j * 32 + 4 * rq;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const int t = 8 * mg + u;
        wv[u] = j < n && t < s ? __ldg(reinterpret_cast<const uint32_t*>(base + t * T.I->rstride)) : 0u;
    }
}
// the words regrouped per entry (4 x 4 byte transposes), 8 bytes per entry into its 128-byte
// swizzled K-major row (K bytes 8 (lane / 8) .. + 7)
__device__ __forceinline__ void crt_tile_store(uint8_t* sA, const uint32_t (&wv)[8]) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rq = lane & 7, mg = lane >> 3;
    uint32_t lo[4], hi[4];
    transpose4(wv[0], wv[1], wv[2], wv[3], lo);
    transpose4(wv[4], wv[5], wv[6], wv[7], hi);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int e = 32 * warp + 4 * rq + u;
        const int c = mg >> 1;  // 16-byte chunk of the 32 K bytes
        *reinterpret_cast<uint2*>(sA + e * 128 + ((c ^ (e & 7)) << 4) + 8 * (mg & 1)) = make_uint2(lo[u], hi[u]);
    }
}

// Software-pipelined over the CTA's tiles: while the MMA of tile k runs, the threads load tile
// k + 1's residues into registers and finish tile k - 1 from the other accumulator (two A tiles,
// two 64-column accumulators, two barriers).
template <int NL>
__global__ void __launch_bounds__(128) crt_mma_kernel(const __grid_constant__ CrtMmaParams P) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t{1023});
    uint8_t* sA0 = smem;                      // two 128 rows x 128 B tiles, K-major, 128-byte swizzle
    uint8_t* sB = smem + 2 * 128 * 128;       // kCrtN rows x 128 B
    uint64_t* bar = reinterpret_cast<uint64_t*>(sB + kCrtN * 128);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 2);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x < kCrtN) {  // B: the W bytes of the plan (only the 32 K bytes of each row are read)
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
        dev::tmem_alloc(dev::smem_addr(tmem_slot), 2 * kCrtN);
        dev::tmem_relinquish();
    }
    dev::tc_fence_before();
    __syncthreads();
    dev::tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    int item = 0;
    {  // the item of this CTA's first tile; later tiles only move forward
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
        return TileRef{I, (local % I->iblocks) * 32, (local / I->iblocks) * 4};
    };
    const int64_t ntiles = P.tiles > blockIdx.x ? (P.tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    uint32_t wv[8];
    TileRef cur{}, prev{};
    if (ntiles > 0) {
        cur = tile_ref(blockIdx.x);
        crt_tile_load(cur, P.s, wv);
    }
    bool ok = true;
    for (int64_t kk = 0; kk <= ntiles && ok; ++kk) {
        const int buf = static_cast<int>(kk & 1);
        if (kk < ntiles) {
            crt_tile_store(sA0 + buf * 128 * 128, wv);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        }
        dev::tc_fence_before();
        __syncthreads();
        if (kk < ntiles && threadIdx.x == 0) {
            dev::tc_fence_after();
            dev::mma_i8(tmem + static_cast<uint32_t>(buf * kCrtN),
                        dev::sw128_kmajor_desc(dev::smem_addr(sA0 + buf * 128 * 128)),
                        dev::sw128_kmajor_desc(dev::smem_addr(sB)), kCrtIdesc, 0u);
            dev::tc_commit(dev::smem_addr(bar + buf));
        }
        TileRef nxt{};
        if (kk + 1 < ntiles) {  // the next tile's loads run under this iteration's waits and arithmetic
            nxt = tile_ref(blockIdx.x + (kk + 1) * gridDim.x);
            crt_tile_load(nxt, P.s, wv);
        }
        if (kk > 0) {  // finish tile kk - 1
            const int pb = buf ^ 1;
            const uint32_t parity = static_cast<uint32_t>(((kk - 1) >> 1) & 1);
            const int w_ok = dev::mbar_wait(dev::smem_addr(bar + pb), parity, abort_flag, P.err,
                                            dev::kErrTimeoutAccFull, P.wait_ns) ? 1 : 0;
            if (!__syncthreads_and(w_ok)) {
                ok = false;
                break;
            }
            dev::tc_fence_after();
            uint32_t d0[32], d1[32];
            const uint32_t taddr = tmem + (static_cast<uint32_t>(32 * warp) << 16) + static_cast<uint32_t>(pb * kCrtN);
            dev::tmem_load_32x32(taddr, d0);
            dev::tmem_load_32x32(taddr + 32, d1);
            dev::tmem_load_wait();
            const CrtItem* __restrict__ I = prev.I;
            const int64_t i = prev.i0 + lane, j = prev.j0 + warp;
            if (i < I->m && j < I->n) {
                uint64_t acc[NL];
#pragma unroll
                for (int l = 0; l < NL; ++l) {
                    const uint32_t b0 = 4 * l < 32 ? d0[(4 * l) & 31] : d1[(4 * l) & 31];
                    const uint32_t b1 = 4 * l + 1 < 32 ? d0[(4 * l + 1) & 31] : d1[(4 * l + 1) & 31];
                    const uint32_t b2 = 4 * l + 2 < 32 ? d0[(4 * l + 2) & 31] : d1[(4 * l + 2) & 31];
                    const uint32_t b3 = 4 * l + 3 < 32 ? d0[(4 * l + 3) & 31] : d1[(4 * l + 3) & 31];
                    acc[l] = static_cast<uint64_t>(b0) + (static_cast<uint64_t>(b1) << 8) +
                             (static_cast<uint64_t>(b2) << 16) + (static_cast<uint64_t>(b3) << 24);
                }
                const uint32_t f0 = 4 * NL < 32 ? d0[(4 * NL) & 31] : d1[(4 * NL) & 31];
                const uint32_t f1 = 4 * NL + 1 < 32 ? d0[(4 * NL + 1) & 31] : d1[(4 * NL + 1) & 31];
                const uint32_t uf = (1u << 15) + f0 + (f1 << 8);
                const int64_t q = static_cast<int64_t>(uf >> 16);
                const int tk = I->tk;
                const int Ej = exponent_of(I->maxB[j], tk), De = exponent_of(I->maxA[i], tk);
                const bool nonfinite = De == kNonFinite || Ej == kNonFinite;
                double v = crt_finish<NL>(acc, q, P.M, nonfinite ? 0 : De + Ej);
                if (nonfinite) v = __longlong_as_double(0x7FF8000000000000ll);
                double* cp = I->C + i + j * I->ldc;
                // the reference's unfused alpha*v + beta*c, one rounding per operation
                const double av = __dmul_rn(I->ar, v);
                *cp = I->br == 0.0 ? av : __dadd_rn(av, __dmul_rn(I->br, *cp));
            }
        }
        prev = cur;
        cur = nxt;
    }
    dev::tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        dev::tc_fence_after();
        dev::tmem_dealloc(tmem, 2 * kCrtN);
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
    if (it.mma) {  // tensor-core CRT: tiles of 32 rows x 4 columns
        it.iblocks = ceil_div(it.m, 32);
        return it.m > 0 ? it.iblocks * ceil_div(it.n, 4) : 0;
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
}  // namespace

void launch_crt(const CrtItem* d_items, int count, int64_t blocks, const Plan& plan, bool cplx, int* err,
                cudaStream_t st) {
    if (crt_uses_mma(plan, cplx)) {
        if (count <= 0 || blocks <= 0) return;
        static thread_local CrtMmaParams P;
        P = CrtMmaParams{};
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
        // four CTAs per SM: 4 x 128 of the 512 TMEM columns (and 4 x 41 KB of shared memory)
        const int grid = static_cast<int>(std::min<int64_t>(blocks, static_cast<int64_t>(sm_count()) * 4));
        crt_mma_kernel<8><<<grid, 128, kCrtSmem, st>>>(P);  // crt_uses_mma: 8 limbs only
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
