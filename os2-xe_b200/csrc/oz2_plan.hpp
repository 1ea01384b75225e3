// oz2_plan.hpp - host planning for the Ozaki Scheme II path: modulus sets, the exact
// product M, the bits per scaled element tk, CRT weights, and the per-modulus constants the
// split, GEMM-epilogue and CRT kernels read.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define OZ2_HD __host__ __device__
#else
#define OZ2_HD
#endif

namespace oz2 {

constexpr int kMaxModuli = 24;     // the reference's range of s (Ozaki2::gemm / zgemm)
// The adaptive path (no counterpart in the reference) may go further, to s = 32, with moduli sets
// of its own: tiles whose certified error bound needs more than the 91 bits per element of 24
// moduli run emulated instead of in native FP64.
constexpr int kMaxModuliExt = 32;
constexpr int kBigWords = 8;       // 256-bit host integers
constexpr int kMaxLimbs = 8;       // 32-bit limbs of M for s <= 32
constexpr int kMaxScaleBits = 100;     // tk cap of the reference's plans (s <= 24)
constexpr int kMaxScaleBitsExt = 124;  // tk cap of the extended plans (s = 25..32)
constexpr int kNarrowScaleBits = 62;
// the split's wide offset (2^93 in three 32-bit words) holds |x| <= 2^92; every plan with
// s <= 24 has tk <= 91
constexpr int kWideScaleBits = 92;
// the widest offset (2^125 in four 32-bit words) holds |x| <= 2^124 (extended plans)
constexpr int kNonFinite = -2147483647 - 1;

// 32-bit limbs of M per s: max(2, floor(log2 M / 32) + 1) (ref src/ozaki2_gpu.hpp:55-59, :168)
// a = q b + r for the block and unit indices of a launch (below 2^31, which the host checks for
// every grid): 32-bit division, several times cheaper than the 64-bit one
OZ2_HD inline void divmod_index(int64_t a, int64_t b, int64_t& q, int64_t& r) {
    const uint32_t qq = static_cast<uint32_t>(a) / static_cast<uint32_t>(b);
    q = qq;
    r = a - static_cast<int64_t>(qq) * b;
}

OZ2_HD constexpr int limbs_for(int s) {
    constexpr int t[kMaxModuliExt + 1] = {0, 0, 2, 2, 2, 2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4,
                                          5, 5, 5, 5, 6, 6, 6, 6, 6, 7, 7, 7, 7, 8, 8, 8};
    return t[s];
}

// Constants of one modulus as the kernels use them.
// GEMM sums of at most kExactKB k-blocks of 128 products of int8 residues are bounded by
// kExactSum = 511 * 128 * 128^2 < 2^30, so c + kbias30 < 2^31 and the epilogue's quotient is exact
constexpr int kExactKB = 511;
constexpr uint32_t kExactSum = 511u * 128u * 16384u;

struct ModConst {
    uint32_t m;      // modulus
    uint32_t mu;     // floor(2^32 / m), Barrett
    uint32_t h;      // (m - 1) / 2: residues are kept symmetric in [-h, m-1-h]
    uint32_t koff3;  // (h - 2^62 mod m) mod m: narrow offset (tk <= 62)
    uint32_t koff5;  // (h - 2^93 mod m) mod m: wide offset
    uint32_t koff7;  // (h - 2^125 mod m) mod m: widest offset (extended plans)
    uint32_t kbias;  // m ceil(2^31 / m): c + kbias is in [0, 2^32) for every int32 GEMM sum c
                     // (|c| < 2^31 - 2^21) and congruent to c modulo m
    uint32_t kbias30;  // m ceil(kExactSum / m): c + kbias30 is in [0, 2^31) for every int32 GEMM sum
                       // c of at most kExactKB k-blocks (|c| <= kExactSum) and congruent to c
    uint32_t mx31;     // ceil(2^(32 + mxs) / m): floor(v / m) = umulhi(v, mx31) >> mxs exactly for v < 2^31
    uint32_t mxs;      // 7, or 6 for m < 128 (the moduli of the extended sets from s = 29), where
                       // ceil(2^39 / m) would not fit 32 bits
    uint32_t cb[4];  // bytes 2^(8 l) mod m, l = 0..15, four per word (byte-limb weights)
    uint32_t m32;    // ceil(2^32 / m): floor(v / m) = umulhi(v, m32) exactly for v < 2^24
    // the split's start values 0x4B000000 + (-2^62 mod m), (-2^93 mod m), (-2^125 mod m): as
    // floats, 2^23 plus the offset that cancels the narrow, wide and widest offset integers
    uint32_t foff3, foff5, foff7;
    float finv;   // fl(1 / m)
    float fbias;  // -2^23 fl(1 / m), exact (a power-of-two multiple)
};

struct Plan {
    int s = 0;
    int nl = 0;
    int tk = 0;
    double log2M = 0;
    uint32_t m[kMaxModuliExt] = {};
    uint32_t y[kMaxModuliExt] = {};             // (M/m_t)^-1 mod m_t
    uint32_t W[kMaxModuliExt][kBigWords] = {};  // CRT weights (M/m_t) y_t
    uint32_t M[kBigWords] = {};
    ModConst mc[kMaxModuliExt] = {};            // per-modulus kernel constants (mod_constants)
};

// Returns 0, or 1 (invalid: s out of [2, 24], k < 1, s too small for k), or 5 (overflow).
// ref src/ozaki2_gpu.hpp:159-200
int make_plan(int s, int64_t k, Plan& p);
// the same for s in [2, 32]: the reference's plans for s <= 24, the extended sets above
int make_plan_ext(int s, int64_t k, Plan& p);
// tk of make_plan_ext(s, k), or 0 where that plan is invalid (s too small for k)
int plan_tk(int s, int64_t k);
const char* plan_error_text(int s, int64_t k, int status, char* buf, int len);

void mod_constants(const Plan& p, ModConst* out);

// CRT table: Sum_t r_t W_t - q M with q = round(Sum_t r_t y_t / m_t) from an estimate whose
// error is far below 1/4 (ref src/ozaki2_gpu.hpp:526-588 uses FP32; here 24-bit fixed point)
constexpr int kQuads = (kMaxModuliExt + 3) / 4;  // moduli in groups of four (one residue byte each)

struct CrtConst {
    int s, nl;
    uint32_t M[kMaxLimbs];
    // W_t = (M / m_t) y_t in 16-bit limbs, paired for two-way byte dot products: for the moduli
    // 4g..4g+3 and limb l, Wq[g][l][0] = W16[4g][l] | W16[4g+1][l] << 16 and Wq[g][l][1] the same
    // for 4g+2, 4g+3 (zero past s)
    uint32_t Wq[kQuads][2 * kMaxLimbs][2];
    // F16_t = min(round(y_t / m_t 2^16), 2^16 - 1), paired the same way: fixed-point quotient
    // weights (error per term below 2^-16, so for s <= 32 the quotient estimate is off by less than
    // 1/8, inside the 1/4 margin that |x| <= M/4 leaves)
    uint32_t Fq[kQuads][2];
};
void crt_constants(const Plan& p, CrtConst& out);

}  // namespace oz2
