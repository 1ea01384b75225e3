// oz2_plan.cpp - see oz2_plan.hpp.
#include "oz2_plan.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

namespace oz2 {
namespace {

// Pairwise-coprime moduli <= 256 for s = 2..24 (ref src/coprime_tables.hpp:10-111): each set
// is a prefix of one of three sequences.
constexpr uint16_t kSeqSmall[6] = {256, 255, 253, 251, 247, 241};
constexpr uint16_t kSeqMid[13] = {256, 253, 251, 249, 247, 245, 241, 239, 233, 229, 227, 223, 211};
constexpr uint16_t kSeqLarge[24] = {256, 253, 251, 249, 247, 241, 239, 235, 233, 229, 227, 223,
                                    217, 211, 199, 197, 193, 191, 181, 179, 173, 167, 163, 157};
// Extended sets (s = 25..32, the adaptive path only; no counterpart in the reference): prefixes of
// the greedy sequence of pairwise-coprime integers <= 256 taken from the top (each the largest
// one coprime with all before it), so M grows by the most a further modulus can give.
constexpr uint16_t kSeqExt[32] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193,
                                  191, 181, 179, 173, 167, 163, 157, 151, 149, 139, 137, 131, 127, 113, 109, 107};

struct Big {
    uint32_t w[kBigWords] = {};
    static Big of(uint64_t v) {
        Big b;
        b.w[0] = static_cast<uint32_t>(v);
        b.w[1] = static_cast<uint32_t>(v >> 32);
        return b;
    }
    bool mul(uint32_t f) {  // false on overflow
        uint64_t c = 0;
        for (auto& x : w) {
            const uint64_t t = uint64_t{x} * f + c;
            x = static_cast<uint32_t>(t);
            c = t >> 32;
        }
        return c == 0;
    }
    uint32_t divmod(uint32_t d) {
        uint64_t r = 0;
        for (int i = kBigWords - 1; i >= 0; --i) {
            const uint64_t cur = (r << 32) | w[i];
            w[i] = static_cast<uint32_t>(cur / d);
            r = cur % d;
        }
        return static_cast<uint32_t>(r);
    }
    uint32_t mod(uint32_t d) const {
        Big t = *this;
        return t.divmod(d);
    }
    bool shl(int bits) {  // false if set bits would be shifted out
        Big r;
        for (int b = kBigWords * 32 - 1; b >= 0; --b) {
            if (!((w[b / 32] >> (b % 32)) & 1u)) continue;
            if (b + bits >= kBigWords * 32) return false;
            r.w[(b + bits) / 32] |= 1u << ((b + bits) % 32);
        }
        *this = r;
        return true;
    }
    int cmp(const Big& o) const {
        for (int i = kBigWords - 1; i >= 0; --i)
            if (w[i] != o.w[i]) return w[i] < o.w[i] ? -1 : 1;
        return 0;
    }
    // estimate from the top three words; the tk search below starts from it
    double log2() const {
        int top = kBigWords - 1;
        while (top > 0 && w[top] == 0) --top;
        const int lo = top - 2 > 0 ? top - 2 : 0;
        double v = 0;
        for (int i = top; i >= lo; --i) v = v * 4294967296.0 + w[i];
        return std::log2(v) + 32.0 * lo;
    }
};

int64_t inverse_mod(int64_t a, int64_t m) {
    int64_t t = 0, nt = 1, r = m, nr = ((a % m) + m) % m;
    while (nr) {
        const int64_t q = r / nr;
        int64_t tmp = t - q * nt;
        t = nt;
        nt = tmp;
        tmp = r - q * nr;
        r = nr;
        nr = tmp;
    }
    return r == 1 ? (t % m + m) % m : -1;
}

uint32_t pow2_mod(int e, uint32_t m) {
    uint32_t v = 1 % m;
    for (int i = 0; i < e; ++i) v = (v * 2) % m;
    return v;
}

}  // namespace

namespace {
// everything of a plan but tk depends on s alone: built once per s
struct Templates {
    Plan plan[kMaxModuliExt + 1];
    int status[kMaxModuliExt + 1];
    Templates() {
        for (int s = 2; s <= kMaxModuliExt; ++s) status[s] = build(s, plan[s]);
    }
    static int build(int s, Plan& p) {
        p = Plan{};
        p.s = s;
        const uint16_t* seq = s <= 6 ? kSeqSmall : (s <= 13 ? kSeqMid : (s <= kMaxModuli ? kSeqLarge : kSeqExt));
        Big M = Big::of(1);
        for (int t = 0; t < s; ++t) {
            p.m[t] = seq[t];
            if (seq[t] != 256 && seq[t] % 2 == 0) return 3;  // the split's rounded quotient needs odd m
            if (!M.mul(seq[t])) return 5;
        }
        p.log2M = M.log2();
        p.nl = static_cast<int>(std::floor(p.log2M / 32.0)) + 1;
        if (p.nl < 2) p.nl = 2;
        if (p.nl != limbs_for(s)) return 3;
        for (int t = 0; t < s; ++t) {
            Big Mt = M;
            if (Mt.divmod(p.m[t]) != 0) return 3;
            const int64_t y = inverse_mod(Mt.mod(p.m[t]), p.m[t]);
            if (y < 0) return 3;
            if (!Mt.mul(static_cast<uint32_t>(y))) return 5;
            std::memcpy(p.W[t], Mt.w, sizeof Mt.w);
            p.y[t] = static_cast<uint32_t>(y);
        }
        std::memcpy(p.M, M.w, sizeof M.w);
        mod_constants(p, p.mc);
        return 0;
    }
};
const Templates& templates() {
    static const Templates t;  // thread-safe initialisation
    return t;
}
}  // namespace

// floor(M / 2^e) for e >= 0, or 2^64 - 1 when that does not fit 64 bits
static uint64_t shr_saturated(const Big& M, int e) {
    for (int i = kBigWords - 1; i >= 0; --i) {
        if (!M.w[i]) continue;
        if (32 * i + 31 - __builtin_clz(M.w[i]) >= e + 64) return ~uint64_t{0};
        break;
    }
    uint64_t r = 0;
    for (int i = 0; i < kBigWords; ++i) {
        const int sh = 32 * i - e;  // where bit 0 of word i lands
        if (!M.w[i] || sh <= -32) continue;
        r |= sh >= 0 ? uint64_t{M.w[i]} << sh : uint64_t{M.w[i]} >> -sh;
    }
    return r;
}

int plan_tk(int s, int64_t k) {
    if (s < 2 || s > kMaxModuliExt || k < 1) return 0;
    const Templates& T = templates();
    if (T.status[s]) return 0;
    const Plan& p = T.plan[s];
    Big M;
    std::memcpy(M.w, p.M, sizeof M.w);
    // largest tk <= 100 (124 for the extended sets) with k 2^(2 tk + 2) <= M, so that |x| <= M/4 for
    // every result entry
    int tk = static_cast<int>(std::floor((p.log2M - 2.0 - std::log2(static_cast<double>(k))) / 2.0));
    const int cap = s <= kMaxModuli ? kMaxScaleBits : kMaxScaleBitsExt;
    if (tk > cap) tk = cap;
    for (;; --tk) {
        if (tk < 1) return 0;
        // k 2^e <= M exactly when k <= floor(M / 2^e), M shifted right by e and saturated to 64 bits
        if (static_cast<uint64_t>(k) <= shr_saturated(M, 2 * tk + 2)) return tk;
    }
}

int make_plan_ext(int s, int64_t k, Plan& p) {
    if (s < 2 || s > kMaxModuliExt || k < 1) return 1;
    const Templates& T = templates();
    if (T.status[s]) return T.status[s];
    const int tk = plan_tk(s, k);
    if (tk < 1) return 1;
    // never for the tables above: the largest tk is 91 at s = 24 and 118 at s = 32
    if (tk > (s <= kMaxModuli ? kWideScaleBits : kMaxScaleBitsExt)) return 5;
    p = T.plan[s];
    p.tk = tk;
    return 0;
}

int make_plan(int s, int64_t k, Plan& p) {
    if (s < 2 || s > kMaxModuli || k < 1) return 1;
    return make_plan_ext(s, k, p);
}

const char* plan_error_text(int s, int64_t k, int status, char* buf, int len) {
    if (s < 2 || s > kMaxModuli)
        std::snprintf(buf, len, "oz2: num_moduli must be in [2, %d]", kMaxModuli);
    else if (k < 1)
        std::snprintf(buf, len, "oz2: k must be >= 1");
    else if (status == 1)
        std::snprintf(buf, len, "oz2: num_moduli=%d is too small for k=%lld", s, static_cast<long long>(k));
    else if (status == 5)
        std::snprintf(buf, len, "oz2: integer overflow while planning");
    else
        std::snprintf(buf, len, "oz2: inconsistent modulus table");
    return buf;
}

void mod_constants(const Plan& p, ModConst* out) {
    for (int t = 0; t < p.s; ++t) {
        const uint32_t m = p.m[t], h = (m - 1) / 2;
        ModConst& c = out[t];
        c.m = m;
        c.mu = static_cast<uint32_t>((uint64_t{1} << 32) / m);
        c.h = h;
        c.koff3 = (h + m - pow2_mod(62, m)) % m;
        c.koff5 = (h + m - pow2_mod(93, m)) % m;
        c.koff7 = (h + m - pow2_mod(125, m)) % m;
        c.kbias = m * static_cast<uint32_t>(((uint64_t{1} << 31) + m - 1) / m);
        c.kbias30 = m * ((kExactSum + m - 1) / m);
        // Granlund and Montgomery (1994): with M = ceil(2^(32 + x) / m) = (2^(32 + x) + e) / m, e < m,
        // floor(v M / 2^(32 + x)) = floor(v / m) for every v < 2^31 when v e < 2^(32 + x), which
        // x = 7 gives for m <= 256 and x = 6 for m < 128 (e <= 126); M fits 32 bits for m > 128
        // with x = 7 and for m > 64 with x = 6
        c.mxs = m > 128 ? 7u : 6u;
        c.mx31 = static_cast<uint32_t>(((uint64_t{1} << (32 + c.mxs)) + m - 1) / m);
        for (int w = 0; w < 4; ++w) {
            c.cb[w] = 0;
            for (int b = 0; b < 4; ++b) c.cb[w] |= pow2_mod(8 * (4 * w + b), m) << (8 * b);
        }
        // division by a constant with an exact multiply-high (Granlund and Montgomery, 1994):
        // with M = ceil(2^32 / m) = (2^32 + e) / m, 0 <= e < m <= 2^8, floor(v M / 2^32) =
        // floor(v / m) for every v < 2^24 (the added v e / (m 2^32) stays below 1 / m)
        c.m32 = static_cast<uint32_t>(((uint64_t{1} << 32) + m - 1) / m);
        c.foff3 = 0x4B000000u + (m - pow2_mod(62, m)) % m;
        c.foff5 = 0x4B000000u + (m - pow2_mod(93, m)) % m;
        c.foff7 = 0x4B000000u + (m - pow2_mod(125, m)) % m;
        c.finv = 1.0f / static_cast<float>(m);
        c.fbias = -8388608.0f * c.finv;
    }
}

void crt_constants(const Plan& p, CrtConst& out) {
    out = CrtConst{};
    out.s = p.s;
    out.nl = p.nl;
    for (int t = 0; t < p.s; ++t) {
        const int g = t / 4, half = (t / 2) & 1, sh = 16 * (t & 1);
        for (int l = 0; l < 2 * p.nl; ++l) {
            const uint32_t w16 = (p.W[t][l / 2] >> (16 * (l & 1))) & 0xFFFFu;
            out.Wq[g][l][half] |= w16 << sh;
        }
        const uint64_t f = ((static_cast<uint64_t>(p.y[t]) << 16) + p.m[t] / 2) / p.m[t];
        out.Fq[g][half] |= static_cast<uint32_t>(std::min<uint64_t>(f, 0xFFFFu)) << sh;
    }
    for (int l = 0; l < p.nl; ++l) out.M[l] = p.M[l];
}

}  // namespace oz2
