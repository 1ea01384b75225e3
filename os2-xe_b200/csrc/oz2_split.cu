// oz2_split.cu - scale and split phases of the Ozaki-II path.
//
// scale: max |x| per plane row as raw FP64 bits (ref src/ozaki2_gpu.hpp:309-358); the bit
//        pattern of a non-negative double orders like the value, and Inf/NaN land above
//        0x7FF0000000000000 so one integer max also detects non-finite rows.
// split: for every element x of plane row r, the integer RNE(x * 2^e_r) with
//        e_r = tk - frexp_exp(max_r) (ref :360-377, :251-289) and its symmetric residue
//        modulo each m_t in [-h_t, m_t-1-h_t] (ref :407-455, complex 3M form :457-520),
//        stored as int8 in the pre-tiled plane layout of oz2_kernels.cuh.
#include "oz2_kernels.cuh"

namespace oz2 {
namespace {

constexpr uint64_t kAbsMask = 0x7FFFFFFFFFFFFFFFull;
constexpr uint32_t kMask21 = 0x1FFFFFu;

__device__ __forceinline__ int exponent_of(unsigned long long b, int tk) {
    if (b >= 0x7FF0000000000000ull) return kNonFinite;
    if (b == 0) return 0;
    const int be = static_cast<int>(b >> 52);
    const int e2 = be ? be - 1022 : -1010 - __clzll(static_cast<long long>(b));  // frexp exponent
    return tk - e2;
}

// ------------------------------------------------------------------ scale
struct ScaleParams {
    const double* X;
    int64_t ldx, rows, k, kchunk;
    unsigned long long* out;
};

// plane rows contiguous in memory: one thread per row, a k range per grid row
template <bool CPLX>
__global__ void __launch_bounds__(256) scale_rowc_kernel(const __grid_constant__ ScaleParams P) {
    const int64_t r = static_cast<int64_t>(blockIdx.x) * 256 + threadIdx.x;
    if (r >= P.rows) return;
    const int64_t p0 = static_cast<int64_t>(blockIdx.y) * P.kchunk;
    const int64_t p1 = min(P.k, p0 + P.kchunk);
    unsigned long long best = 0;
    const unsigned long long* X = reinterpret_cast<const unsigned long long*>(P.X);
    for (int64_t p = p0; p < p1; ++p) {
        const int64_t idx = r + p * P.ldx;
        if (CPLX) {
            best = max(best, X[2 * idx] & kAbsMask);
            best = max(best, X[2 * idx + 1] & kAbsMask);
        } else {
            best = max(best, __ldg(X + idx) & kAbsMask);
        }
    }
    if (best) atomicMax(P.out + r, best);
}

// inner index contiguous: one warp per row, a k range per grid row
template <bool CPLX>
__global__ void __launch_bounds__(256) scale_kc_kernel(const __grid_constant__ ScaleParams P) {
    const int64_t r = static_cast<int64_t>(blockIdx.x) * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= P.rows) return;
    const int w = CPLX ? 2 : 1;
    const int64_t p0 = static_cast<int64_t>(blockIdx.y) * P.kchunk * w;
    const int64_t p1 = min(P.k * w, p0 + P.kchunk * w);
    const unsigned long long* X = reinterpret_cast<const unsigned long long*>(P.X) + r * P.ldx * w;
    unsigned long long best = 0;
    for (int64_t p = p0 + lane; p < p1; p += 32) best = max(best, __ldg(X + p) & kAbsMask);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xFFFFFFFFu, best, o));
    if (lane == 0 && best) atomicMax(P.out + r, best);
}

// ------------------------------------------------------------------ split
struct SplitParams {
    const double* X;
    int64_t ldx, rows, k;
    const unsigned long long* maxbits;
    int tk, s, conj;
    int8_t* planes;
    int64_t plane_bytes, kb_total, rows_pad;
    ModConst mc[kMaxModuli];
};

// 21-bit limbs of 2^OFF + RNE(v 2^e) (OFF = 62 for NLIMB = 3, 104 for NLIMB = 5)
template <int NLIMB>
__device__ __forceinline__ void offset_limbs(double v, int e, uint32_t (&L)[NLIMB]) {
    const uint64_t bits = static_cast<uint64_t>(__double_as_longlong(v));
    const bool neg = (bits >> 63) != 0;
    const int be = static_cast<int>((bits >> 52) & 0x7FF);
    uint64_t mant = bits & 0xFFFFFFFFFFFFFull;
    if (be) mant |= 0x10000000000000ull;
    const int sh = (be ? be : 1) - 1075 + e;
    uint64_t lo = 0, hi = 0;
    if (mant) {
        if (sh >= 0) {
            if (NLIMB == 3) {
                lo = mant << sh;
            } else {
                lo = sh < 64 ? mant << sh : 0;
                hi = sh == 0 ? 0 : (sh < 64 ? mant >> (64 - sh) : mant << (sh - 64));
            }
        } else if (sh >= -54) {
            const int rs = -sh;
            const uint64_t q = mant >> rs;
            const uint64_t rem = mant & ((1ull << rs) - 1);
            const uint64_t half = 1ull << (rs - 1);
            lo = q + ((rem > half || (rem == half && (q & 1))) ? 1 : 0);
        }
    }
    if (NLIMB == 3) {
        const uint64_t xo = neg ? (1ull << 62) - lo : (1ull << 62) + lo;
        L[0] = static_cast<uint32_t>(xo) & kMask21;
        L[1] = static_cast<uint32_t>(xo >> 21) & kMask21;
        L[2] = static_cast<uint32_t>(xo >> 42) & kMask21;
    } else {
        uint64_t ol, oh;
        if (neg) {
            ol = 0 - lo;
            oh = (1ull << 40) - hi - (lo != 0 ? 1 : 0);
        } else {
            ol = lo;
            oh = (1ull << 40) + hi;
        }
        L[0] = static_cast<uint32_t>(ol) & kMask21;
        L[1] = static_cast<uint32_t>(ol >> 21) & kMask21;
        L[2] = static_cast<uint32_t>(ol >> 42) & kMask21;
        L[NLIMB > 3 ? 3 : 0] = static_cast<uint32_t>((ol >> 63) | (oh << 1)) & kMask21;
        L[NLIMB > 4 ? 4 : 0] = static_cast<uint32_t>(oh >> 20) & kMask21;
    }
}

// 2^k as a double for k in [-1022, 1023]
__device__ __forceinline__ double pow2(int k) {
    return __longlong_as_double(static_cast<long long>(k + 1023) << 52);
}

// Narrow path (tk <= 62) in floating point: y = v 2^e as two exact power-of-two products
// (e = e1 + e2 keeps both factors normal for every e this path produces; a product that
// underflows means |y| < 2^-1022, which rounds to 0 like the exact value), then one
// round-to-nearest-even conversion to int64: the same integer as the bit-level RNE above.
__device__ __forceinline__ void offset_limbs_fp(double v, double s1, double s2, uint32_t (&L)[3]) {
    const long long x = __double2ll_rn((v * s1) * s2);
    const uint64_t xo = static_cast<uint64_t>(x + (1ll << 62));
    L[0] = static_cast<uint32_t>(xo) & kMask21;
    L[1] = static_cast<uint32_t>(xo >> 21) & kMask21;
    L[2] = static_cast<uint32_t>(xo >> 42) & kMask21;
}

// symmetric residue of the value whose offset limbs are L, as an int in [-h, m-1-h]
template <int NLIMB>
__device__ __forceinline__ int sym_residue(const uint32_t (&L)[NLIMB], const ModConst& c) {
    uint32_t v = L[0] + (NLIMB == 3 ? c.koff3 : c.koff5);
#pragma unroll
    for (int j = 1; j < NLIMB; ++j) v += L[j] * c.c[j - 1];
    const uint32_t q = __umulhi(v, c.mu);
    uint32_t r = v - q * c.m;
    r = min(r, r - c.m);
    return static_cast<int>(r) - static_cast<int>(c.h);
}

// low bytes of a, b, c, d as one little-endian word
__device__ __forceinline__ uint32_t pack_bytes(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    return __byte_perm(__byte_perm(a, b, 0x0040), __byte_perm(c, d, 0x0040), 0x5410);
}

// Each thread: one plane row r and 16 consecutive inner indices k0..k0+15, i.e. one 16-byte
// chunk of every plane. ROWC: a warp is 32 consecutive rows (coalesced loads along r), the 8
// warps of a block are the 8 chunks of one 128-wide k block. Otherwise a warp is one row and
// 32 consecutive chunks (512 inner indices), the 8 warps are 8 rows.
template <int NLIMB, bool CPLX, bool ROWC>
__global__ void __launch_bounds__(256) split_kernel(const __grid_constant__ SplitParams P) {
    int64_t r, k0;
    if (ROWC) {
        r = static_cast<int64_t>(blockIdx.x) * 32 + (threadIdx.x & 31);
        k0 = static_cast<int64_t>(blockIdx.y) * kTileK + (threadIdx.x >> 5) * 16;
    } else {
        r = static_cast<int64_t>(blockIdx.x) * 8 + (threadIdx.x >> 5);
        k0 = static_cast<int64_t>(blockIdx.y) * (4 * kTileK) + (threadIdx.x & 31) * 16;
    }
    if (r >= P.rows_pad || k0 >= P.kb_total * kTileK) return;
    const int e = r < P.rows ? exponent_of(P.maxbits[r], P.tk) : 0;
    const bool live = r < P.rows && e != kNonFinite;

    constexpr int NG = CPLX ? 2 : 1;
    uint32_t L[NG][16][NLIMB];
    const int e1 = e >> 1;
    const double s1 = pow2(live ? e1 : 0), s2 = pow2(live ? e - e1 : 0);
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int64_t p = k0 + q;
        double v0 = 0.0, v1 = 0.0;
        if (live && p < P.k) {
            const int64_t idx = ROWC ? r + p * P.ldx : p + r * P.ldx;
            if (CPLX) {
                v0 = __ldg(P.X + 2 * idx);
                v1 = __ldg(P.X + 2 * idx + 1);
                if (P.conj) v1 = -v1;  // residues of -y are the negated residues of y
            } else {
                v0 = __ldg(P.X + idx);
            }
        }
        if constexpr (NLIMB == 3) {
            offset_limbs_fp(v0, s1, s2, L[0][q]);
            if (CPLX) offset_limbs_fp(v1, s1, s2, L[NG - 1][q]);
        } else {
            offset_limbs<NLIMB>(v0, e, L[0][q]);
            if (CPLX) offset_limbs<NLIMB>(v1, e, L[NG - 1][q]);
        }
    }

    const int64_t rb = r >> 7;
    const int rr = static_cast<int>(r & 127);
    const int64_t kb = k0 >> 7;
    const int c = static_cast<int>((k0 >> 4) & 7);
    int8_t* out = P.planes + (rb * P.kb_total + kb) * kTileBytes + rr * kTileK + ((c ^ (rr & 7)) << 4);
    const int64_t gstride = static_cast<int64_t>(P.s) * P.plane_bytes;

    for (int t = 0; t < P.s; ++t) {
        const ModConst mc = P.mc[t];
        uint32_t b0[16], b1[16], b2[16];  // residue bytes in the low 8 bits
        if (mc.m == 256) {
            // 2^21 j = 0 mod 256 and 2^62 = 0 mod 256: the residue byte is the low byte of 2^62 + x
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                b0[q] = L[0][q][0];
                if (CPLX) {
                    b1[q] = L[NG - 1][q][0];
                    b2[q] = b0[q] + b1[q];
                }
            }
        } else {
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int s0 = sym_residue<NLIMB>(L[0][q], mc);
                b0[q] = static_cast<uint32_t>(s0);
                if (CPLX) {
                    const int s1 = sym_residue<NLIMB>(L[NG - 1][q], mc);
                    const int m = static_cast<int>(mc.m), h = static_cast<int>(mc.h);
                    int ss = s0 + s1;
                    ss = ss > m - 1 - h ? ss - m : ss;
                    ss = ss < -h ? ss + m : ss;
                    b1[q] = static_cast<uint32_t>(s1);
                    b2[q] = static_cast<uint32_t>(ss);
                }
            }
        }
        uint32_t w0[4], w1[4], w2[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            w0[q] = pack_bytes(b0[4 * q], b0[4 * q + 1], b0[4 * q + 2], b0[4 * q + 3]);
            if (CPLX) {
                w1[q] = pack_bytes(b1[4 * q], b1[4 * q + 1], b1[4 * q + 2], b1[4 * q + 3]);
                w2[q] = pack_bytes(b2[4 * q], b2[4 * q + 1], b2[4 * q + 2], b2[4 * q + 3]);
            }
        }
        *reinterpret_cast<uint4*>(out + t * P.plane_bytes) = make_uint4(w0[0], w0[1], w0[2], w0[3]);
        if (CPLX) {
            *reinterpret_cast<uint4*>(out + gstride + t * P.plane_bytes) = make_uint4(w1[0], w1[1], w1[2], w1[3]);
            *reinterpret_cast<uint4*>(out + 2 * gstride + t * P.plane_bytes) =
                make_uint4(w2[0], w2[1], w2[2], w2[3]);
        }
    }
}

template <int NLIMB, bool CPLX>
void split_dispatch(const SplitParams& P, bool rowc, cudaStream_t st) {
    if (rowc) {
        dim3 grid(static_cast<unsigned>(ceil_div(P.rows_pad, 32)), static_cast<unsigned>(P.kb_total));
        split_kernel<NLIMB, CPLX, true><<<grid, 256, 0, st>>>(P);
    } else {
        dim3 grid(static_cast<unsigned>(ceil_div(P.rows_pad, 8)), static_cast<unsigned>(ceil_div(P.kb_total, 4)));
        split_kernel<NLIMB, CPLX, false><<<grid, 256, 0, st>>>(P);
    }
}

}  // namespace

void launch_scale(const SideDesc& sd, unsigned long long* maxbits, int num_sms, cudaStream_t st) {
    if (sd.rows <= 0 || sd.k <= 0) return;
    ScaleParams P{sd.X, sd.ldx, sd.rows, sd.k, 0, maxbits};
    const int64_t target = static_cast<int64_t>(num_sms) * 2048 * 2;  // threads in flight
    if (sd.row_contig) {
        const int64_t rthreads = round_up(sd.rows, 256);
        int64_t chunks = std::max<int64_t>(1, std::min<int64_t>(sd.k, target / rthreads));
        chunks = std::min<int64_t>(chunks, 65535);
        P.kchunk = ceil_div(sd.k, chunks);
        dim3 grid(static_cast<unsigned>(rthreads / 256), static_cast<unsigned>(ceil_div(sd.k, P.kchunk)));
        if (sd.cplx) scale_rowc_kernel<true><<<grid, 256, 0, st>>>(P);
        else scale_rowc_kernel<false><<<grid, 256, 0, st>>>(P);
    } else {
        const int64_t rthreads = sd.rows * 32;
        int64_t chunks = std::max<int64_t>(1, std::min<int64_t>(ceil_div(sd.k, 256), target / rthreads));
        chunks = std::min<int64_t>(chunks, 65535);
        P.kchunk = ceil_div(sd.k, chunks);
        dim3 grid(static_cast<unsigned>(ceil_div(sd.rows, 8)), static_cast<unsigned>(ceil_div(sd.k, P.kchunk)));
        if (sd.cplx) scale_kc_kernel<true><<<grid, 256, 0, st>>>(P);
        else scale_kc_kernel<false><<<grid, 256, 0, st>>>(P);
    }
}

void launch_split(const SideDesc& sd, const unsigned long long* maxbits, int tk, const ModConst* mc, int s,
                  int8_t* planes, const PlaneGeom& g, cudaStream_t st) {
    SplitParams P{};
    P.X = sd.X;
    P.ldx = sd.ldx;
    P.rows = sd.rows;
    P.k = sd.k;
    P.maxbits = maxbits;
    P.tk = tk;
    P.s = s;
    P.conj = sd.conj ? 1 : 0;
    P.planes = planes;
    P.plane_bytes = g.plane_bytes;
    P.kb_total = g.kb_total;
    P.rows_pad = g.rows_pad;
    for (int t = 0; t < s; ++t) P.mc[t] = mc[t];
    const bool wide = tk > kNarrowScaleBits;
    if (sd.cplx) {
        if (wide) split_dispatch<5, true>(P, sd.row_contig, st);
        else split_dispatch<3, true>(P, sd.row_contig, st);
    } else {
        if (wide) split_dispatch<5, false>(P, sd.row_contig, st);
        else split_dispatch<3, false>(P, sd.row_contig, st);
    }
}

}  // namespace oz2
