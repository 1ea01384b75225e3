// oz2_split.cu - scale and split phases of the Ozaki-II path.
//
// scale: max |x| per plane row as raw FP64 bits (ref src/ozaki2_gpu.hpp:309-358); the bit
//        pattern of a non-negative double orders like the value, and Inf/NaN land above
//        0x7FF0000000000000 so one integer max also detects non-finite rows.
// split: for every element x of plane row r, the integer RNE(x * 2^e_r) with
//        e_r = tk - frexp_exp(max_r) (ref :360-377, :251-289) and its symmetric residue
//        modulo each m_t in [-h_t, m_t-1-h_t] (ref :407-455, complex 3M form :457-520),
//        stored as int8 in the pre-tiled plane layout of oz2_kernels.cuh.
#include <algorithm>
#include <atomic>

#include "oz2_kernels.cuh"
#include "oz2_ptx.cuh"

namespace oz2 {
namespace {

constexpr uint64_t kAbsMask = 0x7FFFFFFFFFFFFFFFull;

__device__ __forceinline__ int exponent_of(unsigned long long b, int tk) {
    if (b >= 0x7FF0000000000000ull) return kNonFinite;
    if (b == 0) return 0;
    const int be = static_cast<int>(b >> 52);
    const int e2 = be ? be - 1022 : -1010 - __clzll(static_cast<long long>(b));  // frexp exponent
    return tk - e2;
}

// ------------------------------------------------------------------ item lookup
// index of the item whose [block0, next block0) range holds `b` (items sorted by block0)
template <class Item>
__device__ __forceinline__ int find_item(const Item* items, int count, int64_t b) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].block0 <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// ------------------------------------------------------------------ scale
// ROWC: plane rows contiguous in memory, one thread per row and a k range per block.
// Otherwise: inner index contiguous, one warp per row and a k range per block.
template <bool CPLX, bool ROWC>
__global__ void __launch_bounds__(256) scale_kernel(const ScaleItem* __restrict__ items, int count) {
    const ScaleItem* I = items + find_item(items, count, blockIdx.x);
    const int64_t local = static_cast<int64_t>(blockIdx.x) - I->block0;
    int64_t rb, kc;
    divmod_index(local, I->rblocks, kc, rb);
    const unsigned long long* X = reinterpret_cast<const unsigned long long*>(I->X);
    const int64_t rows = I->rows, k = I->k, ldx = I->ldx, kchunk = I->kchunk;
    if (ROWC) {
        // 32 consecutive rows per block (one per lane); the 8 warps interleave the k range
        const int64_t r = rb * 32 + (threadIdx.x & 31);
        if (r >= rows) return;
        const int64_t p0 = kc * kchunk, p1 = min(k, p0 + kchunk);
        unsigned long long best = 0;
        for (int64_t p = p0 + (threadIdx.x >> 5); p < p1; p += 8) {
            const int64_t idx = r + p * ldx;
            if (CPLX) {
                best = max(best, __ldg(X + 2 * idx) & kAbsMask);
                best = max(best, __ldg(X + 2 * idx + 1) & kAbsMask);
            } else {
                best = max(best, __ldg(X + idx) & kAbsMask);
            }
        }
        if (best) atomicMax(I->out + r, best);
    } else {
        const int64_t r = rb * 8 + (threadIdx.x >> 5);
        const int lane = threadIdx.x & 31;
        if (r >= rows) return;
        const int w = CPLX ? 2 : 1;
        const int64_t p0 = kc * kchunk * w, p1 = min(k * w, p0 + kchunk * w);
        const unsigned long long* row = X + r * ldx * w;
        unsigned long long best = 0;
        for (int64_t p = p0 + lane; p < p1; p += 32) best = max(best, __ldg(row + p) & kAbsMask);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xFFFFFFFFu, best, o));
        if (lane == 0 && best) atomicMax(I->out + r, best);
    }
}

// ------------------------------------------------------------------ split
// 2^k as a double for k in [-1022, 1023]
__device__ __forceinline__ double pow2(int k) {
    return __longlong_as_double(static_cast<long long>(k + 1023) << 52);
}

// x = RNE(v 2^e) as the reference derives it from the double's bits (src/ozaki2_gpu.hpp:251-289),
// computed in floating point: y = v 2^e as two exact power-of-two products (e = e1 + e2 keeps
// both factors normal for every e the split sees; a product that underflows means
// |y| < 2^-1022, which rounds to 0 like the exact value), then one round-to-nearest-even
// conversion. The offset integer 2^62 + x (narrow path, tk <= 62: x fits int64) as two 32-bit
// words.
__device__ __forceinline__ void offset_words_fp(double v, double s1, double s2, uint32_t (&W)[2]) {
    const long long x = __double2ll_rn((v * s1) * s2);
    const uint64_t xo = static_cast<uint64_t>(x + (1ll << 62));
    W[0] = static_cast<uint32_t>(xo);
    W[1] = static_cast<uint32_t>(xo >> 32);
}

// Wide path (62 < tk <= 92; the largest tk of any plan is 91): y = v 2^e as above, a = |rint(y)|
// <= 2^92 split exactly into hi = trunc(a 2^-64) and lo = a - hi 2^64 (both exact: power-of-two
// scaling, and lo keeps a subset of a's 53 significant bits), then 2^93 +- (hi:lo), which lies in
// (0, 2^94), as three 32-bit words.
__device__ __forceinline__ void offset_words_fp_wide(double v, double s1, double s2, uint32_t (&W)[3]) {
    const double y = rint((v * s1) * s2);
    const double a = fabs(y);
    const double hd = trunc(a * 5.421010862427522e-20);     // 2^-64
    const double ld = fma(hd, -18446744073709551616.0, a);  // a - hd 2^64, exact
    const uint64_t hi = __double2ull_rz(hd), lo = __double2ull_rz(ld);
    uint64_t ol, oh;
    if (y < 0.0) {
        ol = 0 - lo;
        oh = (1ull << 29) - hi - (lo != 0 ? 1 : 0);
    } else {
        ol = lo;
        oh = (1ull << 29) + hi;
    }
    W[0] = static_cast<uint32_t>(ol);
    W[1] = static_cast<uint32_t>(ol >> 32);
    W[2] = static_cast<uint32_t>(oh);
}

// Widest path (92 < tk <= 124, the extended moduli sets of the adaptive path): as the wide path
// with a = |rint(y)| <= 2^124, hi = trunc(a 2^-64) < 2^60, and the offset 2^125 +- (hi:lo), which
// lies in (0, 2^126), as four 32-bit words.
__device__ __forceinline__ void offset_words_fp_widest(double v, double s1, double s2, uint32_t (&W)[4]) {
    const double y = rint((v * s1) * s2);
    const double a = fabs(y);
    const double hd = trunc(a * 5.421010862427522e-20);     // 2^-64
    const double ld = fma(hd, -18446744073709551616.0, a);  // a - hd 2^64, exact
    const uint64_t hi = __double2ull_rz(hd), lo = __double2ull_rz(ld);
    uint64_t ol, oh;
    if (y < 0.0) {
        ol = 0 - lo;
        oh = (1ull << 61) - hi - (lo != 0 ? 1 : 0);
    } else {
        ol = lo;
        oh = (1ull << 61) + hi;
    }
    W[0] = static_cast<uint32_t>(ol);
    W[1] = static_cast<uint32_t>(ol >> 32);
    W[2] = static_cast<uint32_t>(oh);
    W[3] = static_cast<uint32_t>(oh >> 32);
}

// The byte dot products of the offset integer: v = 0x4B000000 + koff + sum_l byte_l (2^(8 l) mod m)
// with koff = -2^62 (-2^93, -2^125) mod m, so that v' = v - 0x4B000000 is congruent to x modulo m
// and below 2^20 (at most 16 bytes: m + 16 255^2), and v's bits are the float 2^23 + v' exactly.
template <int NW>
__device__ __forceinline__ uint32_t byte_dot(const uint32_t (&W)[NW], const ModConst& c) {
    uint32_t v = NW == 2 ? c.foff3 : (NW == 3 ? c.foff5 : c.foff7);
#pragma unroll
    for (int j = 0; j < NW; ++j) v = __dp4a(W[j], c.cb[j], v);
    return v;
}

// The symmetric residue v' - q m, q = rint(v' / m), in [-h, h] (m odd), in the low byte of the
// result (the upper bytes hold a constant of m). One FMA gives fl(v' fl(1/m)): its addend -2^23
// fl(1/m) cancels the 2^23 of v's float exactly, so only the product and one rounding err, by at
// most (v'/m) 2^-23 < 2^-2 / m for v' < 2^21. For odd m, v'/m lies at least 1 / (2m) from every
// half-integer, so adding 1.5 2^23 (round to nearest, ulp 1) gives the float 1.5 2^23 + q with
// bits 0x4B400000 + q. Then v - bits m = v' - q m + (0x4B000000 - 0x4B400000 m), and both
// constants are 0 modulo 256. Per residue: two FP32 operations in place of the integer
// multiply-high quotient, and no shift of [0, m) to [-h, m-1-h] afterwards.
__device__ __forceinline__ uint32_t sym_residue(uint32_t v, const ModConst& c) {
    const float t = __fadd_rn(__fmaf_rn(__uint_as_float(v), c.finv, c.fbias), 12582912.0f);
    return v - __float_as_uint(t) * c.m;
}

// low bytes of a, b, c, d as one little-endian word
__device__ __forceinline__ uint32_t pack_bytes(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    return __byte_perm(__byte_perm(a, b, 0x0040), __byte_perm(c, d, 0x0040), 0x5410);
}

// NLIMB: 3 selects the narrow path (two words per offset integer), 5 the wide one (three words),
// 7 the widest (four words; real operands only: the complex path keeps s <= 24).
// Elements per thread: 16 (one 16-byte chunk of every plane) on the real narrow path; 8 (half a
// chunk) on the wide path (16 measured no faster) and for complex inputs (two groups of words)
constexpr int kSplitRowcK = 256;  // inner indices per block of the rows-contiguous split

template <int NLIMB, bool CPLX>
__host__ __device__ constexpr int split_ept() {
    return NLIMB == 3 && !CPLX ? 16 : 8;
}

// Each thread: one plane row r and EPT consecutive inner indices k0..k0+EPT-1 of every plane.
// Block (bx, by) and thread -> plane row r and the first k0 of its EPT consecutive inner indices.
// ROWC: a warp is EPT consecutive rows times 32 / EPT consecutive EPT-wide pieces: the loads along
// r stay coalesced (EPT rows of 8 bytes per inner index), and the lanes of one row cover 32
// inner indices, a whole 32-byte sector of each plane row (two 16-byte chunks that the swizzle
// keeps adjacent); the 8 warps of a block continue along the inner index, so a block is EPT rows
// by 256 inner indices. Otherwise a warp is one row and 32 consecutive pieces, the 8 warps are 8
// rows.
template <int EPT, bool ROWC>
__device__ __forceinline__ void split_coords(int64_t bx, int64_t by, int64_t& r, int64_t& k0) {
    const int lane = static_cast<int>(threadIdx.x & 31), warp = static_cast<int>(threadIdx.x >> 5);
    if (ROWC) {
        r = bx * EPT + lane % EPT;
        k0 = by * kSplitRowcK + (warp * (32 / EPT) + lane / EPT) * EPT;
    } else {
        r = bx * 8 + warp;
        k0 = by * (32 * EPT) + lane * EPT;
    }
}

// The EPT elements (r, k0 .. k0 + EPT - 1) of every plane, r < rows_pad and k0 < the padded k:
// maxb is the row's maximum bits (read only for r < rows).
template <int NLIMB, bool CPLX, bool ROWC>
__device__ __forceinline__ void split_piece(const SplitItem* __restrict__ I, int64_t r, int64_t k0,
                                            unsigned long long maxb) {
    constexpr int EPT = split_ept<NLIMB, CPLX>();
    const int64_t kb_total = I->kb_total, plane_bytes = I->plane_bytes, ldx = I->ldx, k = I->k;
    const int64_t rows = I->rows;
    const double* X = I->X;
    const int conj = I->conj, nmod = I->s;
    const int64_t rb = r >> 7;
    const int rr = static_cast<int>(r & 127);
    const int64_t kb = k0 >> 7;
    const int c = static_cast<int>((k0 >> 4) & 7);
    int8_t* out = I->planes + (rb * kb_total + kb) * kTileBytes + rr * kTileK + ((c ^ (rr & 7)) << 4) +
                  (k0 & 15);  // the second half of a chunk on the wide path
    const int64_t gstride = static_cast<int64_t>(nmod) * plane_bytes;
    auto store = [&](int8_t* dst, const uint32_t (&w)[EPT / 4]) {
        if constexpr (EPT == 16) *reinterpret_cast<uint4*>(dst) = make_uint4(w[0], w[1], w[2], w[3]);
        else *reinterpret_cast<uint2*>(dst) = make_uint2(w[0], w[1]);
    };
    if (r >= rows || k0 >= k) {  // padding: residues of zero are zero
        const uint32_t z[EPT / 4] = {};
        for (int t = 0; t < nmod; ++t) {
            store(out + t * plane_bytes, z);
            if (CPLX) {
                store(out + gstride + t * plane_bytes, z);
                store(out + 2 * gstride + t * plane_bytes, z);
            }
        }
        return;
    }
    const int e = exponent_of(maxb, I->tk);
    const bool live = e != kNonFinite;

    constexpr int NG = CPLX ? 2 : 1;
    constexpr int NW = NLIMB == 3 ? 2 : (NLIMB == 5 ? 3 : 4);  // 32-bit words of the offset integer
    uint32_t L[NG][EPT][NW];
    const int e1 = e >> 1;
    const double s1 = pow2(live ? e1 : 0), s2 = pow2(live ? e - e1 : 0);
#pragma unroll
    for (int q = 0; q < EPT; ++q) {
        const int64_t p = k0 + q;
        double v0 = 0.0, v1 = 0.0;
        if (live && p < k) {
            const int64_t idx = ROWC ? r + p * ldx : p + r * ldx;
            if (CPLX) {
                v0 = __ldg(X + 2 * idx);
                v1 = __ldg(X + 2 * idx + 1);
                if (conj) v1 = -v1;  // residues of -y are the negated residues of y
            } else {
                v0 = __ldg(X + idx);
            }
        }
        if constexpr (NLIMB == 3) {
            offset_words_fp(v0, s1, s2, L[0][q]);
            if (CPLX) offset_words_fp(v1, s1, s2, L[NG - 1][q]);
        } else if constexpr (NLIMB == 5) {
            offset_words_fp_wide(v0, s1, s2, L[0][q]);
            if (CPLX) offset_words_fp_wide(v1, s1, s2, L[NG - 1][q]);
        } else {
            offset_words_fp_widest(v0, s1, s2, L[0][q]);
        }
    }

    // real operands: two moduli per pass, so one modulus's constant loads and dot products overlap
    // the other's (measured 2-12 % faster over the narrow, wide and widest paths; the complex path,
    // whose registers are already high, measured slower with it)
#pragma unroll(CPLX ? 1 : 2)
    for (int t = 0; t < nmod; ++t) {
        const ModConst mc = I->mc[t];
        uint32_t b0[EPT], b1[EPT], b2[EPT];  // residue bytes in the low 8 bits
        if (mc.m == 256) {
            // 2^62 = 2^93 = 2^125 = 0 mod 256: the residue byte is the low byte of the offset integer
#pragma unroll
            for (int q = 0; q < EPT; ++q) {
                b0[q] = L[0][q][0];
                if (CPLX) {
                    b1[q] = L[NG - 1][q][0];
                    b2[q] = b0[q] + b1[q];
                }
            }
        } else {
#pragma unroll
            for (int q = 0; q < EPT; ++q) {
                const uint32_t v0 = byte_dot<NW>(L[0][q], mc);
                b0[q] = sym_residue(v0, mc);
                if (CPLX) {
                    const uint32_t v1 = byte_dot<NW>(L[NG - 1][q], mc);
                    b1[q] = sym_residue(v1, mc);
                    b2[q] = sym_residue(v0 + v1 - 0x4B000000u, mc);  // x0 + x1: v0' + v1' < 2^21
                }
            }
        }
        // the residue bytes (as int8), four per word
        uint32_t w0[EPT / 4], w1[EPT / 4], w2[EPT / 4];
#pragma unroll
        for (int q = 0; q < EPT / 4; ++q) {
            w0[q] = pack_bytes(b0[4 * q], b0[4 * q + 1], b0[4 * q + 2], b0[4 * q + 3]);
            if (CPLX) {
                w1[q] = pack_bytes(b1[4 * q], b1[4 * q + 1], b1[4 * q + 2], b1[4 * q + 3]);
                w2[q] = pack_bytes(b2[4 * q], b2[4 * q + 1], b2[4 * q + 2], b2[4 * q + 3]);
            }
        }
        store(out + t * plane_bytes, w0);
        if (CPLX) {
            store(out + gstride + t * plane_bytes, w1);
            store(out + 2 * gstride + t * plane_bytes, w2);
        }
    }
}

template <int NLIMB, bool CPLX, bool ROWC>
__device__ __forceinline__ void split_block(const SplitItem* __restrict__ items, int count) {
    constexpr int EPT = split_ept<NLIMB, CPLX>();
    const SplitItem* __restrict__ I = items + find_item(items, count, blockIdx.x);
    const int64_t local = static_cast<int64_t>(blockIdx.x) - I->block0;
    int64_t bx, by;
    divmod_index(local, I->rblocks, by, bx);
    int64_t r, k0;
    split_coords<EPT, ROWC>(bx, by, r, k0);
    if (r >= I->rows_pad || k0 >= I->kb_total * kTileK) return;
    split_piece<NLIMB, CPLX, ROWC>(I, r, k0, r < I->rows && k0 < I->k ? I->maxbits[r] : 0ull);
}

// Real operands: registers capped for three blocks of 256 per SM on the narrow path (16 elements
// per thread, 80 registers) and four on the wide and widest paths (8 elements per thread, 64
// registers, no spills). Complex operands keep the compiler's own allocation (two blocks per SM).
template <int NLIMB, bool ROWC>
__global__ void __launch_bounds__(256, NLIMB == 3 ? 3 : 4) split_kernel(const SplitItem* __restrict__ items, int count) {
    split_block<NLIMB, false, ROWC>(items, count);
}

template <int NLIMB, bool ROWC>
__global__ void __launch_bounds__(256) split_kernel_cplx(const SplitItem* __restrict__ items, int count) {
    split_block<NLIMB, true, ROWC>(items, count);
}

// ------------------------------------------------------------------ scale fused into the split
// One launch for both phases of a real operand (ref src/ozaki2_gpu.hpp:974-989 then :1004-1022
// run them as two passes over A and B): a block owns whole plane rows, takes their maxima over
// all of k (and writes them for the CRT), then splits the same rows. The second read of the rows
// follows the first within the block, so it is served by L2 while the rows that all resident
// blocks have in flight fit there (the launcher uses it for k up to kFuseMaxK: at most 8 rows of
// 16 KiB, or 16 rows of 4 KiB, per block). k contiguous: 8 rows per block, a warp per row, lanes
// over k. Rows contiguous: EPT rows per block (a 128-byte line per inner index), the 256 / EPT
// thread groups over k, then the split's own warp layout over 256-wide k blocks.
template <int NLIMB, bool ROWC>
__global__ void __launch_bounds__(256) scale_split_kernel(const SplitItem* __restrict__ items, int count) {
    constexpr int EPT = split_ept<NLIMB, false>();
    constexpr int RB = ROWC ? EPT : 8;  // rows per block
    __shared__ unsigned long long smax[RB];
    const SplitItem* __restrict__ I = items + find_item(items, count, blockIdx.x);
    const int64_t r0 = (static_cast<int64_t>(blockIdx.x) - I->block0) * RB;
    const unsigned long long* X = reinterpret_cast<const unsigned long long*>(I->X);
    const int64_t rows = I->rows, k = I->k, ldx = I->ldx, kpad = I->kb_total * kTileK;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < RB) smax[tid] = 0;
    __syncthreads();
    if (ROWC) {
        const int64_t r = r0 + tid % RB;
        unsigned long long best = 0;
        if (r < rows) {
#pragma unroll 4
            for (int64_t p = tid / RB; p < k; p += 256 / RB) best = max(best, __ldg(X + r + p * ldx) & kAbsMask);
        }
        if (best) atomicMax(&smax[tid % RB], best);
    } else {
        const int64_t r = r0 + warp;
        unsigned long long best = 0;
        if (r < rows) {
#pragma unroll 4
            for (int64_t p = lane; p < k; p += 32) best = max(best, __ldg(X + p + r * ldx) & kAbsMask);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xFFFFFFFFu, best, o));
        if (lane == 0) smax[warp] = best;
    }
    __syncthreads();
    if (tid < RB && r0 + tid < rows) const_cast<unsigned long long*>(I->maxbits)[r0 + tid] = smax[tid];  // for the CRT
    if (ROWC) {
        for (int64_t by = 0; by * kSplitRowcK < kpad; ++by) {
            int64_t r, k0;
            split_coords<EPT, true>(blockIdx.x - I->block0, by, r, k0);  // bx: this block's EPT rows
            if (r < I->rows_pad && k0 < kpad) split_piece<NLIMB, false, true>(I, r, k0, smax[r - r0]);
        }
    } else {
        const int64_t r = r0 + warp;
        if (r < I->rows_pad)
            for (int64_t k0 = lane * EPT; k0 < kpad; k0 += 32 * EPT) split_piece<NLIMB, false, false>(I, r, k0, smax[warp]);
    }
}

// ------------------------------------------------------------------ tensor-core split
// The byte dot products of byte_residue, v_t = Sum_l byte_l (2^(8 l) mod m_t), form a small
// matrix product: (moduli x bytes) times (bytes x elements). One tcgen05.mma kind::i8 (unsigned
// A and B, M = 128, N = 256, K = 32, int32 in TMEM) computes them for a unit of 512 elements:
//   B (N x K, K-major): column n holds two elements, segment g = 0, 1 in bytes 16 g .. 16 g + 15
//     (the offset integer's 8 / 12 / 16 bytes, zero-filled);
//   A (M x K, K-major): row 32 q + l is the slot sigma = 32 (q % Qa) + l, sigma < 2 s: segment
//     sigma / s, modulus sigma % s, the weights 2^(8 l) mod m in that segment's bytes. With
//     Qa = 1 (s <= 16) all four TMEM lane quarters hold the same 32 slots, with Qa = 2 (s <= 32)
//     quarters 0, 1 hold the 2 s slots and 2, 3 repeat them, so every epilogue warp reads its own
//     lane quarter (a hardware rule) and the quarters split the 256 columns between them.
// The epilogue turns v + koff into the residue (x + h) mod m by the exact multiply-high quotient
// (v < 2^20), subtracts h modulo 256 and stores the 32 residues of one slot's 32 consecutive
// inner indices as one 32-byte piece of its plane. The integer pipe keeps one multiply-high and
// one multiply-subtract per residue; the dp4a of byte_residue move to the tensor core.
// Persistent, one CTA per SM with 16 warps, software-pipelined over the CTA's units: while the
// MMA of unit k runs, the threads finish unit k - 1 from the other accumulator (two A and two B
// tiles, 2 x 256 TMEM columns); a unit's FP64 loads are issued kTcAhead units ahead, into
// registers.
constexpr int kTcThreads = 512;
constexpr int kTcAhead = 3;
constexpr int kTcSmem = 1024 + 2 * 16384 + 2 * 32768 + 64;  // two A tiles, two B tiles, barriers + TMEM slot
constexpr int kTcSmemLaunch = 160 * 1024;                   // one CTA per SM (TMEM: 2 x 256 columns)
constexpr uint32_t kTcIdesc = (2u << 4)                     // D: s32; A, B: unsigned 8-bit, K-major
                              | (static_cast<uint32_t>(256 >> 3) << 17) | (static_cast<uint32_t>(128 >> 4) << 24);

template <bool ROWC>
struct TcGeom {
    static constexpr int UR = ROWC ? 16 : 4;    // rows per unit
    static constexpr int UK = ROWC ? 32 : 128;  // inner indices per unit
    // element f = 0..511 of a unit -> row offset, inner offset (loads: coalesced along the
    // contiguous index), segment and column
    __device__ static void element(int f, int& ro, int& po, int& seg, int& n) {
        if (ROWC) {
            ro = f & 15;
            po = f >> 4;
            seg = ro >> 3;
            n = ((ro & 7) << 5) | po;
        } else {
            ro = f >> 7;
            po = f & 127;
            seg = ro >> 1;
            n = ((ro & 1) << 7) | po;
        }
    }
    // the 32 columns n0 .. n0 + 31 of segment seg -> row offset and first inner offset
    __device__ static void chunk(int seg, int n0, int& ro, int& po) {
        if (ROWC) {
            ro = 8 * seg + (n0 >> 5);
            po = 0;
        } else {
            ro = 2 * seg + (n0 >> 7);
            po = n0 & 127;
        }
    }
};

template <int NW>
__device__ __forceinline__ void offset_words(double v, double s1, double s2, uint32_t (&W)[4]) {
    if constexpr (NW == 2) {
        uint32_t w[2];
        offset_words_fp(v, s1, s2, w);
        W[0] = w[0], W[1] = w[1], W[2] = 0, W[3] = 0;
    } else if constexpr (NW == 3) {
        uint32_t w[3];
        offset_words_fp_wide(v, s1, s2, w);
        W[0] = w[0], W[1] = w[1], W[2] = w[2], W[3] = 0;
    } else {
        offset_words_fp_widest(v, s1, s2, W);
    }
}

template <int NW, bool ROWC>
__global__ void __launch_bounds__(kTcThreads, 1) split_tc_kernel(const SplitItem* __restrict__ items, int count,
                                                                int64_t units, int* err) {
    using G = TcGeom<ROWC>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t{1023});
    uint8_t* sA0 = smem;              // two 128 rows x 128 bytes (swizzled; the first two chunks used)
    uint8_t* sB0 = smem + 2 * 16384;  // two 256 rows x 128 bytes
    uint64_t* bar_p = reinterpret_cast<uint64_t*>(smem + 2 * 16384 + 2 * 32768);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar_p + 2);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        dev::mbar_init(dev::smem_addr(bar_p), 1);
        dev::mbar_init(dev::smem_addr(bar_p + 1), 1);
        *abort_flag = 0;
        dev::fence_barrier_init();
    }
    if (warp == 0) {
        dev::tmem_alloc(dev::smem_addr(tmem_slot), 512);
        dev::tmem_relinquish();
    }
    dev::tc_fence_before();
    __syncthreads();
    dev::tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int64_t stride = gridDim.x;
    const int64_t nmine = units > blockIdx.x ? (units - 1 - blockIdx.x) / stride + 1 : 0;
    int ro_l, po_l, seg_l, n_l;  // this thread's element of every unit
    G::element(tid, ro_l, po_l, seg_l, n_l);

    int first = 0;
    {  // the item of this CTA's first unit; later units only move forward
        int hi = count - 1;
        const int64_t u = blockIdx.x;
        while (first < hi) {
            const int mid = (first + hi + 1) >> 1;
            if (items[mid].block0 <= u) first = mid;
            else hi = mid - 1;
        }
    }
    auto advance = [&](int& cur, int64_t u) {
        while (cur + 1 < count && items[cur + 1].block0 <= u) ++cur;
    };
    // the element's value (0 outside the item's rows and k, and for non-finite rows, whose
    // residues are then zero like the padding's) and its row's maximum bits
    int cur_l = first;
    auto load_elem = [&](int64_t kk, double& v, unsigned long long& mb) {
        v = 0.0;
        mb = 0;
        if (kk >= nmine) return;
        const int64_t u = blockIdx.x + kk * stride;
        advance(cur_l, u);
        const SplitItem* I = items + cur_l;
        const int64_t local = u - I->block0;
        int64_t qd, rm;
        divmod_index(local, I->rblocks, qd, rm);
        const int64_t r = rm * G::UR + ro_l, p = qd * G::UK + po_l;
        if (r < I->rows && p < I->k) {
            mb = __ldg(I->maxbits + r);
            if (mb < 0x7FF0000000000000ull) v = __ldg(I->X + (ROWC ? r + p * I->ldx : p + r * I->ldx));
        }
    };
    double pv[kTcAhead];
    unsigned long long pm[kTcAhead];
#pragma unroll
    for (int a = 0; a < kTcAhead; ++a) load_elem(a, pv[a], pm[a]);

    int cur_w = first, cur_e = first;  // items of the unit being written and of the one being finished
    int a_item0 = -1, a_item1 = -1;    // item whose weights are in A tile 0 / 1
    int e_item = -1;                   // item of the epilogue lane constants
    bool valid = false;
    int seg = 0, qa = 1;
    uint32_t m = 1, m32 = 0, koff = 0, c256h = 0;
    int8_t* plane = nullptr;
    bool ok = true;
    uint32_t committed = 0, last_par = 0;  // (thread 0) per accumulator: a commit issued, its parity
    for (int64_t kb = 0; ok && kb <= nmine; kb += kTcAhead) {
#pragma unroll
        for (int a = 0; a < kTcAhead; ++a) {
            const int64_t kk = kb + a;  // unit kk is written, unit kk - 1 finished
            if (!ok || kk > nmine) break;
            const int buf = static_cast<int>(kk & 1);
            if (kk < nmine) {
                const int64_t u = blockIdx.x + kk * stride;
                advance(cur_w, u);
                const SplitItem* __restrict__ I = items + cur_w;
                if ((buf ? a_item1 : a_item0) != cur_w) {  // unit kk - 2's MMA, this tile's last reader, is complete
                    if (buf) a_item1 = cur_w;
                    else a_item0 = cur_w;
                    if (tid < 128) {
                        const int s = I->s, q2 = s <= 16 ? 1 : 2;
                        const int sigma = 32 * ((tid >> 5) % q2) + (tid & 31);
                        uint4 w0 = make_uint4(0, 0, 0, 0), w1 = w0;
                        if (sigma < 2 * s) {
                            const ModConst& c = I->mc[sigma % s];
                            const uint4 cw = make_uint4(c.cb[0], c.cb[1], NW > 2 ? c.cb[2] : 0u, NW > 3 ? c.cb[3] : 0u);
                            if (sigma < s) w0 = cw;
                            else w1 = cw;
                        }
                        uint8_t* row = sA0 + buf * 16384 + tid * 128;
                        *reinterpret_cast<uint4*>(row + ((0 ^ (tid & 7)) << 4)) = w0;
                        *reinterpret_cast<uint4*>(row + ((1 ^ (tid & 7)) << 4)) = w1;
                    }
                }
                const int e = exponent_of(pm[a], I->tk);
                const bool live = e != kNonFinite;
                const int e1 = e >> 1;
                const double s1 = pow2(live ? e1 : 0), s2 = pow2(live ? e - e1 : 0);
                uint32_t W[4];
                offset_words<NW>(pv[a], s1, s2, W);
                *reinterpret_cast<uint4*>(sB0 + buf * 32768 + n_l * 128 + ((seg_l ^ (n_l & 7)) << 4)) =
                    make_uint4(W[0], W[1], W[2], W[3]);
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            }
            dev::tc_fence_before();
            __syncthreads();
            if (kk < nmine && tid == 0) {
                dev::tc_fence_after();
                dev::mma_i8(tmem + static_cast<uint32_t>(buf * 256), dev::sw128_kmajor_desc(dev::smem_addr(sA0 + buf * 16384)),
                            dev::sw128_kmajor_desc(dev::smem_addr(sB0 + buf * 32768)), kTcIdesc, 0u);
                dev::tc_commit(dev::smem_addr(bar_p + buf));
                committed |= 1u << buf;
                last_par = (last_par & ~(1u << buf)) | (static_cast<uint32_t>((kk >> 1) & 1) << buf);
            }
            if (kk < nmine) load_elem(kk + kTcAhead, pv[a], pm[a]);
            if (kk > 0) {  // finish unit kk - 1
                const int pb = buf ^ 1;
                const uint32_t parity = static_cast<uint32_t>(((kk - 1) >> 1) & 1);
                int got = 1;  // one thread waits; the others sleep in the block barrier
                if (tid == 0)
                    got = dev::mbar_wait(dev::smem_addr(bar_p + pb), parity, abort_flag, err, dev::kErrTimeoutAccFull,
                                         dev::kWaitLimitNs) ? 1 : 0;
                if (!__syncthreads_and(got)) {
                    ok = false;
                    break;
                }
                dev::tc_fence_after();
                const int64_t u = blockIdx.x + (kk - 1) * stride;
                advance(cur_e, u);
                const SplitItem* __restrict__ I = items + cur_e;
                if (cur_e != e_item) {
                    e_item = cur_e;
                    const int s = I->s;
                    qa = s <= 16 ? 1 : 2;
                    const int sigma = 32 * ((warp & 3) % qa) + lane;
                    valid = sigma < 2 * s;
                    if (valid) {
                        const int t = sigma % s;
                        const ModConst& c = I->mc[t];
                        seg = sigma / s;
                        m = c.m;
                        m32 = c.m32;
                        koff = NW == 2 ? c.koff3 : (NW == 3 ? c.koff5 : c.koff7);
                        c256h = 256u - c.h;
                        plane = I->planes + t * I->plane_bytes;
                    }
                }
                const int64_t local = u - I->block0;
                int64_t qd, rm;
                divmod_index(local, I->rblocks, qd, rm);
                const int64_t r0 = rm * G::UR, p0 = qd * G::UK;
                // warp (quarter q, part pt) reads lane quarter q: with qa = 1 (four copies of the
                // slots) 16 columns, with qa = 2 (two copies) 32 columns
                const int q = warp & 3, pt = warp >> 2;
                const uint32_t taddr = tmem + (static_cast<uint32_t>(32 * q) << 16) + static_cast<uint32_t>(pb * 256);
                if (qa == 1) {
                    const int n0 = 16 * (4 * q + pt);
                    uint32_t d[16];
                    dev::tmem_load_32x16(taddr + n0, d);
                    dev::tmem_load_wait();
                    if (valid) {
                        int ro, po;
                        G::chunk(seg, n0 & ~31, ro, po);
                        const int64_t r = r0 + ro, pk = p0 + po + (n0 & 31);
                        const int rr = static_cast<int>(r & 127);
                        const int c = static_cast<int>((pk & 127) >> 4);
                        int8_t* tile = plane + ((r >> 7) * I->kb_total + (pk >> 7)) * kTileBytes + rr * kTileK;
                        uint32_t w[4];
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            uint32_t r4[4];
#pragma unroll
                            for (int b = 0; b < 4; ++b) {
                                const uint32_t v = d[4 * j + b] + koff;     // < 2^20 + 2^8
                                r4[b] = v - __umulhi(v, m32) * m + c256h;  // low byte: (x mod m, symmetric)
                            }
                            w[j] = pack_bytes(r4[0], r4[1], r4[2], r4[3]);
                        }
                        *reinterpret_cast<uint4*>(tile + ((c ^ (rr & 7)) << 4)) = make_uint4(w[0], w[1], w[2], w[3]);
                    }
                } else {
                    const int n0 = 32 * (4 * (q >> 1) + pt);
                    uint32_t d[32];
                    dev::tmem_load_32x32(taddr + n0, d);
                    dev::tmem_load_wait();
                    if (valid) {
                        int ro, po;
                        G::chunk(seg, n0, ro, po);
                        const int64_t r = r0 + ro, pk = p0 + po;
                        const int rr = static_cast<int>(r & 127);
                        const int c = static_cast<int>((pk & 127) >> 4);
                        int8_t* tile = plane + ((r >> 7) * I->kb_total + (pk >> 7)) * kTileBytes + rr * kTileK;
                        uint32_t w[8];
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            uint32_t r4[4];
#pragma unroll
                            for (int b = 0; b < 4; ++b) {
                                const uint32_t v = d[4 * j + b] + koff;
                                r4[b] = v - __umulhi(v, m32) * m + c256h;
                            }
                            w[j] = pack_bytes(r4[0], r4[1], r4[2], r4[3]);
                        }
                        *reinterpret_cast<uint4*>(tile + ((c ^ (rr & 7)) << 4)) = make_uint4(w[0], w[1], w[2], w[3]);
                        *reinterpret_cast<uint4*>(tile + (((c + 1) ^ (rr & 7)) << 4)) = make_uint4(w[4], w[5], w[6], w[7]);
                    }
                }
            }
        }
    }
    if (!ok && tid == 0) {  // the last MMA of each accumulator completes before TMEM is freed
        for (int b = 0; b < 2; ++b)
            if (committed & (1u << b)) dev::mbar_wait_drain(dev::smem_addr(bar_p + b), (last_par >> b) & 1u);
    }
    dev::tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        dev::tc_fence_after();
        dev::tmem_dealloc(tmem, 512);
    }
}

// Ozaki Scheme I digits (the reference's comparison baseline, benchmarks/ozaki1_gpu.hpp:31-40):
// x = RNE(v 2^e) as on the narrow split path (tk = 7L - 2 <= 61), then L balanced base-128
// digits in [-64, 63], most significant in plane 0, written in the same plane layout and with
// the same thread mapping as split_kernel's narrow real path (16 elements per thread).
template <bool ROWC>
__global__ void __launch_bounds__(256) slice_kernel(const SplitItem* __restrict__ items, int count) {
    constexpr int EPT = 16;
    const SplitItem* __restrict__ I = items + find_item(items, count, blockIdx.x);
    const int64_t local = static_cast<int64_t>(blockIdx.x) - I->block0;
    int64_t bx, by;
    divmod_index(local, I->rblocks, by, bx);
    int64_t r, k0;
    split_coords<EPT, ROWC>(bx, by, r, k0);
    const int64_t kb_total = I->kb_total, plane_bytes = I->plane_bytes, ldx = I->ldx, k = I->k;
    if (r >= I->rows_pad || k0 >= kb_total * kTileK) return;
    const int ndig = I->s;
    const int64_t rb = r >> 7;
    const int rr = static_cast<int>(r & 127);
    const int c = static_cast<int>((k0 >> 4) & 7);
    int8_t* out = I->planes + (rb * kb_total + (k0 >> 7)) * kTileBytes + rr * kTileK + ((c ^ (rr & 7)) << 4);
    long long x[EPT];
#pragma unroll
    for (int q = 0; q < EPT; ++q) x[q] = 0;
    if (r < I->rows && k0 < k) {
        const int e = exponent_of(I->maxbits[r], I->tk);
        if (e != kNonFinite) {
            const int e1 = e >> 1;
            const double s1 = pow2(e1), s2 = pow2(e - e1);
#pragma unroll
            for (int q = 0; q < EPT; ++q) {
                const int64_t p = k0 + q;
                if (p < k) x[q] = __double2ll_rn((__ldg(I->X + (ROWC ? r + p * ldx : p + r * ldx)) * s1) * s2);
            }
        }
    }
    // least significant digit first, into planes ndig - 1 .. 0
    for (int i = ndig - 1; i >= 0; --i) {
        uint32_t b[EPT];
#pragma unroll
        for (int q = 0; q < EPT; ++q) {
            const long long d = ((x[q] + 64) & 127) - 64;
            x[q] = (x[q] - d) >> 7;
            b[q] = static_cast<uint32_t>(d);
        }
        uint32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) w[q] = pack_bytes(b[4 * q], b[4 * q + 1], b[4 * q + 2], b[4 * q + 3]);
        *reinterpret_cast<uint4*>(out + i * plane_bytes) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

template <int NW>
void split_tc_dispatch(const SplitItem* d, int count, int64_t units, bool rowc, int* err, cudaStream_t st) {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    const unsigned grid = static_cast<unsigned>(std::min<int64_t>(units, static_cast<int64_t>(sms)));
    if (rowc) split_tc_kernel<NW, true><<<grid, kTcThreads, kTcSmemLaunch, st>>>(d, count, units, err);
    else split_tc_kernel<NW, false><<<grid, kTcThreads, kTcSmemLaunch, st>>>(d, count, units, err);
}

std::atomic<int> g_split_tc{0};
std::atomic<int> g_scale_fusion{0};

template <int NLIMB>
void scale_split_dispatch(const SplitItem* d, int count, int64_t blocks, bool rowc, cudaStream_t st) {
    if (rowc) scale_split_kernel<NLIMB, true><<<static_cast<unsigned>(blocks), 256, 0, st>>>(d, count);
    else scale_split_kernel<NLIMB, false><<<static_cast<unsigned>(blocks), 256, 0, st>>>(d, count);
}

template <int NLIMB, bool CPLX>
void split_dispatch(const SplitItem* d, int count, int64_t blocks, bool rowc, cudaStream_t st) {
    if constexpr (CPLX) {
        if (rowc) split_kernel_cplx<NLIMB, true><<<static_cast<unsigned>(blocks), 256, 0, st>>>(d, count);
        else split_kernel_cplx<NLIMB, false><<<static_cast<unsigned>(blocks), 256, 0, st>>>(d, count);
    } else {
        if (rowc) split_kernel<NLIMB, true><<<static_cast<unsigned>(blocks), 256, 0, st>>>(d, count);
        else split_kernel<NLIMB, false><<<static_cast<unsigned>(blocks), 256, 0, st>>>(d, count);
    }
}

}  // namespace

int64_t scale_item_blocks(ScaleItem& it, int num_sms, int64_t block0) {
    it.block0 = block0;
    if (it.rows <= 0 || it.k <= 0) {
        it.rblocks = 1;
        it.kchunk = 1;
        return 0;
    }
    const int64_t target = static_cast<int64_t>(num_sms) * 2048 * 2;  // threads in flight
    if (it.row_contig) {
        it.rblocks = ceil_div(it.rows, 32);
        // at least 64 inner indices per block (8 per warp)
        const int64_t chunks =
            std::max<int64_t>(1, std::min<int64_t>(ceil_div(it.k, 64), target / (it.rblocks * 256)));
        it.kchunk = ceil_div(it.k, chunks);
    } else {
        it.rblocks = ceil_div(it.rows, 8);
        const int64_t chunks = std::max<int64_t>(1, std::min<int64_t>(ceil_div(it.k, 256), target / (it.rows * 32)));
        it.kchunk = ceil_div(it.k, chunks);
    }
    return it.rblocks * ceil_div(it.k, it.kchunk);
}

int64_t split_item_blocks(SplitItem& it, int64_t block0) {
    it.block0 = block0;
    const int ept = it.tk > kNarrowScaleBits || it.cplx ? split_ept<5, false>() : split_ept<3, false>();
    const int64_t kpad = it.kb_total * kTileK;  // inner indices of the plane, padding included
    if (it.row_contig) {
        it.rblocks = ceil_div(it.rows_pad, ept);
        it.kblocks = ceil_div(kpad, kSplitRowcK);
    } else {
        it.rblocks = ceil_div(it.rows_pad, 8);
        it.kblocks = ceil_div(kpad, 32 * ept);
    }
    return it.rblocks * it.kblocks;
}

int64_t split_geometry(SplitItem& it, int64_t block0) {
    if (it.fuse) {  // whole rows per block
        it.tc = 0;
        it.block0 = block0;
        const int rb = it.row_contig ? (it.tk > kNarrowScaleBits ? 8 : 16) : 8;
        it.rblocks = it.rows_pad / rb;
        it.kblocks = 1;
        return it.rblocks;
    }
    it.tc = !it.cplx && g_split_tc.load() ? 1 : 0;
    if (!it.tc) return split_item_blocks(it, block0);
    it.block0 = block0;
    const int ur = it.row_contig ? TcGeom<true>::UR : TcGeom<false>::UR;
    const int uk = it.row_contig ? TcGeom<true>::UK : TcGeom<false>::UK;
    it.rblocks = it.rows_pad / ur;              // rows_pad is a multiple of 128
    it.kblocks = it.kb_total * (kTileK / uk);
    return it.rblocks * it.kblocks;
}

void set_split_path(int tc) { g_split_tc.store(tc ? 1 : 0); }
void set_scale_fusion(int on) { g_scale_fusion.store(on ? 1 : 0); }
bool fuse_scale(bool cplx, bool row_contig, int64_t k) {
    return g_scale_fusion.load() && !cplx && k > 0 && k <= (row_contig ? kFuseMaxKRowc : kFuseMaxK);
}
int split_path() { return g_split_tc.load(); }

cudaError_t prepare_split_kernels() {
    cudaError_t e = cudaSuccess;
    auto set = [&](const void* f) {
        if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmemLaunch);
    };
    set(reinterpret_cast<const void*>(split_tc_kernel<2, false>));
    set(reinterpret_cast<const void*>(split_tc_kernel<2, true>));
    set(reinterpret_cast<const void*>(split_tc_kernel<3, false>));
    set(reinterpret_cast<const void*>(split_tc_kernel<3, true>));
    set(reinterpret_cast<const void*>(split_tc_kernel<4, false>));
    set(reinterpret_cast<const void*>(split_tc_kernel<4, true>));
    return e;
}

void launch_scale(const ScaleItem* d, const ScaleItem* h, int count, int64_t blocks, cudaStream_t st) {
    if (count <= 0 || blocks <= 0) return;
    const bool rowc = h[0].row_contig != 0, cplx = h[0].cplx != 0;
    const unsigned g = static_cast<unsigned>(blocks);
    if (rowc) {
        if (cplx) scale_kernel<true, true><<<g, 256, 0, st>>>(d, count);
        else scale_kernel<false, true><<<g, 256, 0, st>>>(d, count);
    } else {
        if (cplx) scale_kernel<true, false><<<g, 256, 0, st>>>(d, count);
        else scale_kernel<false, false><<<g, 256, 0, st>>>(d, count);
    }
}

void launch_slice(const SplitItem* d, const SplitItem* h, int count, int64_t blocks, cudaStream_t st) {
    if (count <= 0 || blocks <= 0) return;
    if (h[0].row_contig) slice_kernel<true><<<static_cast<unsigned>(blocks), 256, 0, st>>>(d, count);
    else slice_kernel<false><<<static_cast<unsigned>(blocks), 256, 0, st>>>(d, count);
}

void launch_split(const SplitItem* d, const SplitItem* h, int count, int64_t blocks, int* err, cudaStream_t st) {
    if (count <= 0 || blocks <= 0) return;
    const bool wide = h[0].tk > kNarrowScaleBits, rowc = h[0].row_contig != 0;
    if (h[0].fuse) {
        if (h[0].tk > kWideScaleBits) scale_split_dispatch<7>(d, count, blocks, rowc, st);
        else if (wide) scale_split_dispatch<5>(d, count, blocks, rowc, st);
        else scale_split_dispatch<3>(d, count, blocks, rowc, st);
        return;
    }
    if (h[0].tc) {
        if (h[0].tk > kWideScaleBits) split_tc_dispatch<4>(d, count, blocks, rowc, err, st);
        else if (wide) split_tc_dispatch<3>(d, count, blocks, rowc, err, st);
        else split_tc_dispatch<2>(d, count, blocks, rowc, err, st);
        return;
    }
    if (h[0].tk > kWideScaleBits) {  // extended sets: real operands only
        split_dispatch<7, false>(d, count, blocks, rowc, st);
        return;
    }
    if (h[0].cplx) {
        if (wide) split_dispatch<5, true>(d, count, blocks, rowc, st);
        else split_dispatch<3, true>(d, count, blocks, rowc, st);
    } else {
        if (wide) split_dispatch<5, false>(d, count, blocks, rowc, st);
        else split_dispatch<3, false>(d, count, blocks, rowc, st);
    }
}

}  // namespace oz2
