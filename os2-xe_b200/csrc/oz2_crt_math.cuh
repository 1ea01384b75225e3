// oz2_crt_math.cuh - the exact CRT reconstruction of one C entry, shared by the CRT kernels
// (oz2_crt.cu) and the GEMM whose epilogue runs the CRT for small s (oz2_gemm.cu).
#pragma once

#include <cstdint>

#include "oz2_plan.hpp"

namespace oz2 {

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
// The sums of crt_value for EG entries at once: every weight word is read once and used for all
// of them (the entries' dot products interleave, and a constant costs one load, not EG). uf[e] is
// the rounded quotient sum (q = uf >> 16) and acc[e][l] the limb sums of entry e.
template <int S, int NL, int EG>
__device__ __forceinline__ void crt_sums(const uint32_t (&R)[EG][(S + 3) / 4], const CrtConst& cc,
                                         uint32_t (&uf)[EG], uint64_t (&acc)[EG][NL]) {
    constexpr int Q = (S + 3) / 4;
#pragma unroll
    for (int e = 0; e < EG; ++e) uf[e] = 1u << 15;
#pragma unroll
    for (int g = 0; g < Q; ++g) {
        const uint32_t f0 = cc.Fq[g][0], f1 = cc.Fq[g][1];
#pragma unroll
        for (int e = 0; e < EG; ++e) uf[e] = __dp2a_hi(f1, R[e][g], __dp2a_lo(f0, R[e][g], uf[e]));
    }
#pragma unroll
    for (int l = 0; l < NL; ++l) {
        uint32_t a0[EG], a1[EG];  // 16-bit limbs 2l and 2l + 1
#pragma unroll
        for (int e = 0; e < EG; ++e) a0[e] = a1[e] = 0;
#pragma unroll
        for (int g = 0; g < Q; ++g) {
            const uint32_t w00 = cc.Wq[g][2 * l][0], w01 = cc.Wq[g][2 * l][1];
            const uint32_t w10 = cc.Wq[g][2 * l + 1][0], w11 = cc.Wq[g][2 * l + 1][1];
#pragma unroll
            for (int e = 0; e < EG; ++e) {
                a0[e] = __dp2a_hi(w01, R[e][g], __dp2a_lo(w00, R[e][g], a0[e]));
                a1[e] = __dp2a_hi(w11, R[e][g], __dp2a_lo(w10, R[e][g], a1[e]));
            }
        }
#pragma unroll
        for (int e = 0; e < EG; ++e) acc[e][l] = static_cast<uint64_t>(a0[e]) + (static_cast<uint64_t>(a1[e]) << 16);
    }
}

template <int NL>
__device__ __forceinline__ double crt_finish(const uint64_t (&acc)[NL], int64_t q, const uint32_t* Mw, int shift) {
    // the quotient is below 2^16 (a 16-bit fraction sum shifted by 16), so q M_l is one
    // 32 x 32 -> 64-bit product
    const uint64_t q32 = static_cast<uint32_t>(q);
    uint32_t w[NL];
    int64_t carry = 0;
#pragma unroll
    for (int l = 0; l < NL; ++l) {
        const int64_t v = static_cast<int64_t>(acc[l]) - static_cast<int64_t>(q32 * Mw[l]) + carry;
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
    // magnitude without a branch: (X xor s) + (s & 1) over the words, s all ones when negative
    const uint64_t sgn = static_cast<uint64_t>(static_cast<int64_t>(X[NW - 1]) >> 63);
    uint64_t inc = sgn & 1u;
#pragma unroll
    for (int i = 0; i < NW; ++i) {
        const uint64_t t = (X[i] ^ sgn) + inc;
        inc &= t == 0 ? 1u : 0u;  // the carry goes on only past a word that wrapped to zero
        X[i] = t;
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
    return __longlong_as_double(__double_as_longlong(val) | static_cast<long long>(sgn & 0x8000000000000000ull));
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

}  // namespace oz2
