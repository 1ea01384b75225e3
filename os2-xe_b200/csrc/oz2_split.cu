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

#include "oz2_kernels.cuh"

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
    const int64_t rb = local % I->rblocks, kc = local / I->rblocks;
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

// (x + h) mod m in [0, m) from the bytes of the offset integer: v = koff + sum_l byte_l (2^(8 l)
// mod m) by byte dot products (at most 16 bytes, so v < 255 + 16 255^2 < 2^20), then the exact
// multiply-high quotient by ceil(2^32 / m). Two (three, four) dot products, one multiply-high
// and one multiply-subtract per residue.
template <int NW>
__device__ __forceinline__ uint32_t byte_residue(const uint32_t (&W)[NW], const ModConst& c) {
    uint32_t v = NW == 2 ? c.koff3 : (NW == 3 ? c.koff5 : c.koff7);
#pragma unroll
    for (int j = 0; j < NW; ++j) v = __dp4a(W[j], c.cb[j], v);
    return v - __umulhi(v, c.m32) * c.m;
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

template <int NLIMB, bool CPLX, bool ROWC>
__global__ void __launch_bounds__(256) split_kernel(const SplitItem* __restrict__ items, int count) {
    constexpr int EPT = split_ept<NLIMB, CPLX>();
    const SplitItem* __restrict__ I = items + find_item(items, count, blockIdx.x);
    const int64_t local = static_cast<int64_t>(blockIdx.x) - I->block0;
    const int64_t bx = local % I->rblocks, by = local / I->rblocks;
    int64_t r, k0;
    split_coords<EPT, ROWC>(bx, by, r, k0);
    const int64_t kb_total = I->kb_total, plane_bytes = I->plane_bytes, ldx = I->ldx, k = I->k;
    const int64_t rows = I->rows;
    if (r >= I->rows_pad || k0 >= kb_total * kTileK) return;
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
    const int e = exponent_of(I->maxbits[r], I->tk);
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
                const uint32_t r0 = byte_residue<NW>(L[0][q], mc);
                b0[q] = r0;
                if (CPLX) {
                    const uint32_t r1 = byte_residue<NW>(L[NG - 1][q], mc);
                    // (x0 + x1 + h) mod m from the two shifted residues
                    uint32_t r2 = r0 + r1 + (mc.m - mc.h);
                    r2 = min(r2, r2 - mc.m);
                    r2 = min(r2, r2 - mc.m);
                    b1[q] = r1;
                    b2[q] = r2;
                }
            }
        }
        // bytes r - h modulo 256, four per word (m = 256 stores x mod 256 directly)
        const uint32_t h4 = mc.m == 256 ? 0u : mc.h * 0x01010101u;
        uint32_t w0[EPT / 4], w1[EPT / 4], w2[EPT / 4];
#pragma unroll
        for (int q = 0; q < EPT / 4; ++q) {
            w0[q] = __vsub4(pack_bytes(b0[4 * q], b0[4 * q + 1], b0[4 * q + 2], b0[4 * q + 3]), h4);
            if (CPLX) {
                w1[q] = __vsub4(pack_bytes(b1[4 * q], b1[4 * q + 1], b1[4 * q + 2], b1[4 * q + 3]), h4);
                w2[q] = __vsub4(pack_bytes(b2[4 * q], b2[4 * q + 1], b2[4 * q + 2], b2[4 * q + 3]), h4);
            }
        }
        store(out + t * plane_bytes, w0);
        if (CPLX) {
            store(out + gstride + t * plane_bytes, w1);
            store(out + 2 * gstride + t * plane_bytes, w2);
        }
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
    const int64_t bx = local % I->rblocks, by = local / I->rblocks;
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

template <int NLIMB, bool CPLX>
void split_dispatch(const SplitItem* d, int count, int64_t blocks, bool rowc, cudaStream_t st) {
    if (rowc) split_kernel<NLIMB, CPLX, true><<<static_cast<unsigned>(blocks), 256, 0, st>>>(d, count);
    else split_kernel<NLIMB, CPLX, false><<<static_cast<unsigned>(blocks), 256, 0, st>>>(d, count);
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

void launch_split(const SplitItem* d, const SplitItem* h, int count, int64_t blocks, cudaStream_t st) {
    if (count <= 0 || blocks <= 0) return;
    const bool wide = h[0].tk > kNarrowScaleBits, rowc = h[0].row_contig != 0;
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
