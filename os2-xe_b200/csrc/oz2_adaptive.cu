// oz2_adaptive.cu - device side of the adaptive choice of the number of moduli s per C tile
// (no counterpart in the reference):
//   stats    : per panel of 512 rows of op(A) (columns of op(B)), a histogram of exponent gaps
//              g = e(row max) - e(|x|) over the nonzero elements, and the count of zeros
//   features : per tile, quantiles of both panels' gaps, zero fractions, the spread of row
//              (column) maxima, the tile's rows and columns, log2 k and the target bits, plus the
//              analytic s: the smallest s
//              whose bits per element tk reach R + 2 + t - floor(log2(k - 1)), R the largest
//              gap. Every product term then carries a relative error <= 3 * 2^(R - tk), so
//              |C - AB| <= k 2^-t |A||B| holds entry by entry (the DGEMM-level target); kNativeS
//              (native FP64) where even 32 moduli (the extended sets above 24) do not reach it.
//   probe    : Freivalds-style check of a computed tile, C x against A (B x) in double-double
//              with x = e_j for kProbeCols stratified random columns j: each entry (i, j) of those
//              columns against its own tolerance k 2^-t (|A||B|)_ij plus the rounding of C, so a
//              tile meeting the target always passes.
//   dd_ref / error ratio : double-double products and max_ij |C - AB| / (k 2^-t (|A||B|)_ij),
//              used to label training tiles (the smallest s that meets the target).
#include <cstdint>

#include "oz2_adaptive.cuh"

namespace oz2 {
namespace {

__device__ __forceinline__ int frexp_exp_bits(unsigned long long b) {  // frexp exponent of |x| from bits
    const int be = static_cast<int>((b >> 52) & 0x7FF);
    return be ? be - 1022 : -1010 - __clzll(static_cast<long long>(b));
}

template <class Item>
__device__ __forceinline__ int find_block_item(const Item* items, int count, int64_t b) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].block0 <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// ---------------------------------------------------------------- panel statistics
template <bool ROWC>
__global__ void __launch_bounds__(256) panel_stats_kernel(const StatItem* __restrict__ items, int count) {
    __shared__ unsigned int hist[kGapBins + 1];
    for (int i = threadIdx.x; i <= kGapBins; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    const StatItem* I = items + find_block_item(items, count, blockIdx.x);
    const int64_t local = static_cast<int64_t>(blockIdx.x) - I->block0;
    int64_t rb, kc;
    divmod_index(local, I->rblocks, kc, rb);
    const unsigned long long* X = reinterpret_cast<const unsigned long long*>(I->X);
    const int64_t rows = I->rows, k = I->k, ldx = I->ldx;
    const int64_t p0 = kc * I->kchunk, p1 = min(k, p0 + I->kchunk);
    auto add = [&](unsigned long long bits, int erow) {
        bits &= 0x7FFFFFFFFFFFFFFFull;
        if (bits == 0) {
            atomicAdd(&hist[kGapBins], 1u);
        } else if (bits < 0x7FF0000000000000ull) {
            const int g = min(max(erow - frexp_exp_bits(bits), 0), kGapBins - 1);
            atomicAdd(&hist[g], 1u);
        }
    };
    if (ROWC) {  // 32 rows per block, warps interleave k
        const int64_t r = rb * 32 + (threadIdx.x & 31);
        if (r < rows) {
            const unsigned long long mb = I->maxbits[r];
            if (mb != 0 && mb < 0x7FF0000000000000ull) {
                const int erow = frexp_exp_bits(mb);
                for (int64_t p = p0 + (threadIdx.x >> 5); p < p1; p += 8) add(__ldg(X + r + p * ldx), erow);
            }
        }
    } else {  // 8 rows per block, lanes over k
        const int64_t r = rb * 8 + (threadIdx.x >> 5);
        if (r < rows) {
            const unsigned long long mb = I->maxbits[r];
            if (mb != 0 && mb < 0x7FF0000000000000ull) {
                const int erow = frexp_exp_bits(mb);
                for (int64_t p = p0 + (threadIdx.x & 31); p < p1; p += 32) add(__ldg(X + p + r * ldx), erow);
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i <= kGapBins; i += blockDim.x)
        if (hist[i]) atomicAdd(I->hist + i, hist[i]);
}

// Scale and statistics in one pass over DRAM. ROWC: 32 rows per block (one per lane), the 8 warps
// interleave the inner index, the row maximum is combined through shared memory; otherwise one
// warp per row (8 rows per block), lanes over the inner index. The second read of the rows
// (the histogram against the row maximum) comes from the L2. Same maxima and counts as
// scale_kernel followed by panel_stats_kernel.
template <bool ROWC>
__global__ void __launch_bounds__(256) scale_stats_kernel(const StatItem* __restrict__ items, int count) {
    __shared__ unsigned int hist[kGapBins + 1];
    __shared__ unsigned long long part[8][32];
    for (int i = threadIdx.x; i <= kGapBins; i += blockDim.x) hist[i] = 0;
    const StatItem* I = items + find_block_item(items, count, blockIdx.x);
    const int64_t rb = static_cast<int64_t>(blockIdx.x) - I->block0;
    const unsigned long long* X = reinterpret_cast<const unsigned long long*>(I->X);
    const int64_t rows = I->rows, k = I->k, ldx = I->ldx;
    const int warp = static_cast<int>(threadIdx.x >> 5), lane = static_cast<int>(threadIdx.x & 31);
    auto add = [&](unsigned long long bits, int erow) {
        bits &= 0x7FFFFFFFFFFFFFFFull;
        if (bits == 0) {
            atomicAdd(&hist[kGapBins], 1u);
        } else if (bits < 0x7FF0000000000000ull) {
            const int g = min(max(erow - frexp_exp_bits(bits), 0), kGapBins - 1);
            atomicAdd(&hist[g], 1u);
        }
    };
    unsigned long long mb = 0;  // the row maximum (bits of |x|)
    int64_t r;
    if (ROWC) {
        r = rb * 32 + lane;
        unsigned long long best = 0;
        if (r < rows)
            for (int64_t p = warp; p < k; p += 8) best = max(best, __ldg(X + r + p * ldx) & 0x7FFFFFFFFFFFFFFFull);
        part[warp][lane] = best;
        __syncthreads();
#pragma unroll
        for (int w = 0; w < 8; ++w) mb = max(mb, part[w][lane]);
        if (warp == 0 && r < rows) I->maxbits[r] = mb;
    } else {
        r = rb * 8 + warp;
        unsigned long long best = 0;
        if (r < rows)
            for (int64_t p = lane; p < k; p += 32) best = max(best, __ldg(X + p + r * ldx) & 0x7FFFFFFFFFFFFFFFull);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xFFFFFFFFu, best, o));
        mb = best;
        if (lane == 0 && r < rows) I->maxbits[r] = mb;
        __syncthreads();  // the histogram's zeroing is visible
    }
    if (r < rows && mb != 0 && mb < 0x7FF0000000000000ull) {
        const int erow = frexp_exp_bits(mb);
        if (ROWC) {
            for (int64_t p = warp; p < k; p += 8) add(__ldg(X + r + p * ldx), erow);
        } else {
            for (int64_t p = lane; p < k; p += 32) add(__ldg(X + p + r * ldx), erow);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i <= kGapBins; i += blockDim.x)
        if (hist[i]) atomicAdd(I->hist + i, hist[i]);
}

// ---------------------------------------------------------------- features + analytic s
__device__ float gap_quantile(const unsigned int* h, unsigned long long nonzero, float q) {
    if (nonzero == 0) return 0.0f;
    const unsigned long long want = static_cast<unsigned long long>(q * static_cast<double>(nonzero - 1)) + 1;
    unsigned long long c = 0;
    for (int g = 0; g < kGapBins; ++g) {
        c += h[g];
        if (c >= want) return static_cast<float>(g);
    }
    return static_cast<float>(kGapBins - 1);
}
__device__ int gap_max(const unsigned int* h) {
    for (int g = kGapBins - 1; g >= 0; --g)
        if (h[g]) return g;
    return 0;
}

// e(max) - e(min) over the finite nonzero row maxima of a panel
__device__ float exponent_spread(const unsigned long long* maxbits, int64_t rows) {
    int lo = 1 << 30, hi = -(1 << 30);
    for (int64_t r = 0; r < rows; ++r) {
        const unsigned long long b = maxbits[r];
        if (b == 0 || b >= 0x7FF0000000000000ull) continue;
        const int e = frexp_exp_bits(b);
        lo = min(lo, e);
        hi = max(hi, e);
    }
    return hi >= lo ? static_cast<float>(hi - lo) : 0.0f;
}

__global__ void tile_features_kernel(const FeatureItem* __restrict__ items, int count, float* __restrict__ feat,
                                     int* __restrict__ s_analytic) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const FeatureItem& I = items[t];
    const unsigned int* ha = I.hist_a;
    const unsigned int* hb = I.hist_b;
    unsigned long long na = 0, nb = 0;
    for (int g = 0; g < kGapBins; ++g) {
        na += ha[g];
        nb += hb[g];
    }
    const double ta = static_cast<double>(na + ha[kGapBins]), tb = static_cast<double>(nb + hb[kGapBins]);
    float* f = feat + static_cast<int64_t>(t) * kFeatures;
    f[0] = log2f(static_cast<float>(I.k)) / 16.0f;
    f[1] = static_cast<float>(I.target_bits) / 64.0f;
    const float qs[4] = {0.5f, 0.75f, 0.9f, 0.99f};
    for (int q = 0; q < 4; ++q) {
        f[2 + q] = gap_quantile(ha, na, qs[q]) / 64.0f;
        f[8 + q] = gap_quantile(hb, nb, qs[q]) / 64.0f;
    }
    const int ra = gap_max(ha), rb = gap_max(hb);
    f[6] = ra / 64.0f;
    f[12] = rb / 64.0f;
    f[7] = ta > 0 ? static_cast<float>(ha[kGapBins] / ta) : 0.0f;
    f[13] = tb > 0 ? static_cast<float>(hb[kGapBins] / tb) : 0.0f;
    f[14] = exponent_spread(I.maxbits_a, I.rows_a) / 64.0f;
    f[15] = exponent_spread(I.maxbits_b, I.rows_b) / 64.0f;
    // edge tiles hold fewer rows / columns: fewer entries, other statistics
    f[16] = static_cast<float>(I.rows_a) / 512.0f;
    f[17] = static_cast<float>(I.rows_b) / 512.0f;
    // analytic s: tk >= R + 2 + t - floor(log2(k - 1)); the last gap bin holds every gap of 63 or
    // more, so R = 63 bounds nothing: native FP64
    const int R = max(ra, rb);
    int lg = 0;
    for (int64_t v = I.k - 1; v > 1; v >>= 1) ++lg;
    const int need = R + 2 + I.target_bits - lg;
    int s = kNativeS;  // no moduli set suffices: native FP64
    if (R < kGapBins - 1)
        for (int c = 2; c <= kMaxModuliExt; ++c)
            if (I.tk[c] >= need) {
                s = c;
                break;
            }
    s_analytic[t] = s;
}

// ---------------------------------------------------------------- double-double helpers
struct dd {
    double hi, lo;
};
__device__ __forceinline__ dd two_sum(double a, double b) {
    const double s = a + b;
    const double bb = s - a;
    return {s, (a - (s - bb)) + (b - bb)};
}
__device__ __forceinline__ dd dd_add(dd a, dd b) {
    dd s = two_sum(a.hi, b.hi);
    s.lo += a.lo + b.lo;
    return two_sum(s.hi, s.lo);
}
__device__ __forceinline__ dd dd_add_prod(dd acc, double a, double b) {  // acc + a*b
    const double ph = a * b;
    const double pl = fma(a, b, -ph);
    dd s = two_sum(acc.hi, ph);
    s.lo += acc.lo + pl;
    return two_sum(s.hi, s.lo);
}

// ---------------------------------------------------------------- probe
// One block per (tile, kProbeRows rows of the tile). The probe takes kProbeCols columns j_c of the tile
// (stratified: one random column in each of kProbeCols equal ranges) and checks every entry
// (i, j_c) of its rows on its own: C_ij against alpha (A B)_ij, so the check is entry by entry,
// with no cancellation between columns. (A B)_ij is summed in FP64 in blocks of 32 terms (FMA),
// the block sums added into a second accumulator: its error is at most
// (gamma_32 + gamma_(k/32 + 1) (1 + gamma_32)) (|A||B|)_ij < (34 + k/32) 2^-52 (|A||B|)_ij, far
// below the k 2^-53 (|A||B|)_ij tolerance, and that error is added to the tolerance. A is read
// once per tile. A thread holds two rows (i and i + kProbeThreads) and the chunk of B's columns
// sits in shared memory as [p][column], so one 16-byte shared load feeds eight FP64 FMAs.
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__global__ void __launch_bounds__(kProbeThreads, 3) probe_kernel(const ProbeItem* __restrict__ items, int count,
                                                                 int* __restrict__ fail) {
    constexpr int R = kProbeRowsPerThread, NC = kProbeCols;
    static_assert(NC == 8, "the shared-memory row of B is read as four double2");
    const ProbeItem* I = items + find_block_item(items, count, blockIdx.x);
    const int64_t rblk = static_cast<int64_t>(blockIdx.x) - I->block0;
    const int64_t mt = I->mt, nt = I->nt, k = I->k;
    const int ncol = static_cast<int>(min(static_cast<int64_t>(NC), nt));
    __shared__ int64_t cols[NC];
    __shared__ __align__(16) double bs[kProbeChunk][NC];
    if (threadIdx.x < NC) {
        const int c = threadIdx.x;
        int64_t j = c;
        if (nt >= NC) {
            const int64_t span = nt / NC;
            const uint64_t h = mix64(I->seed ^ static_cast<uint64_t>(c));
            j = c * span + static_cast<int64_t>(h % static_cast<uint64_t>(span));
        }
        cols[c] = j;
    }
    __syncthreads();
    const int64_t i0 = rblk * kProbeRows + threadIdx.x;
    bool live[R];
    const double* Ai[R];
    const int64_t astep = I->a_rowc ? I->lda : 1;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int64_t i = i0 + r * kProbeThreads;
        live[r] = i < mt;
        Ai[r] = I->a_rowc ? I->A + i : I->A + i * I->lda;  // dereferenced only for live rows
    }
    double z[R][NC], zp[R][NC], za[R][NC];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
        for (int c = 0; c < NC; ++c) z[r][c] = zp[r][c] = za[r][c] = 0.0;
    for (int64_t p0 = 0; p0 < k; p0 += kProbeChunk) {
        const int pn = static_cast<int>(min(static_cast<int64_t>(kProbeChunk), k - p0));
        for (int e = threadIdx.x; e < NC * pn; e += blockDim.x) {
            const int c = e / pn, q = e - c * pn;
            double v = 0.0;  // columns beyond nt: never checked
            if (c < ncol) {
                const int64_t j = cols[c], p = p0 + q;
                v = I->b_rowc ? I->B[j + p * I->ldb] : I->B[p + j * I->ldb];
            }
            bs[q][c] = v;
        }
        __syncthreads();
        if (live[0]) {
            for (int q0 = 0; q0 < pn; q0 += 32) {  // kProbeChunk is a multiple of 32
                const int qe = min(q0 + 32, pn);
                for (int q1 = q0; q1 < qe; q1 += 4) {
                    // the next four terms of both rows' loads in flight before their products
                    double av[R][4];
#pragma unroll
                    for (int r = 0; r < R; ++r)
#pragma unroll
                        for (int u = 0; u < 4; ++u)
                            av[r][u] = live[r] && q1 + u < qe ? __ldg(Ai[r] + (p0 + q1 + u) * astep) : 0.0;
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int q = min(q1 + u, pn - 1);  // av = 0 past the chunk
                        const double2* b2 = reinterpret_cast<const double2*>(bs[q]);
                        const double2 b01 = b2[0], b23 = b2[1], b45 = b2[2], b67 = b2[3];
                        const double b[NC] = {b01.x, b01.y, b23.x, b23.y, b45.x, b45.y, b67.x, b67.y};
#pragma unroll
                        for (int r = 0; r < R; ++r)
#pragma unroll
                            for (int c = 0; c < NC; ++c) {
                                zp[r][c] = fma(av[r][u], b[c], zp[r][c]);
                                za[r][c] = fma(fabs(av[r][u]), fabs(b[c]), za[r][c]);
                            }
                    }
                }
#pragma unroll
                for (int r = 0; r < R; ++r)
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        z[r][c] += zp[r][c];
                        zp[r][c] = 0.0;
                    }
            }
        }
        __syncthreads();
    }
    bool bad = false;
    const double kd = static_cast<double>(k);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        if (!live[r]) continue;
        const int64_t i = i0 + r * kProbeThreads;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            if (c < ncol) {
                const double cv = I->C[i + cols[c] * I->ldc];
                // C - alpha z in double-double (alpha z exact as a two-product)
                const dd az{I->alpha * z[r][c], fma(I->alpha, z[r][c], -I->alpha * z[r][c])};
                const dd diff = dd_add(dd{cv, 0.0}, dd{-az.hi, -az.lo});
                const double err = fabs(diff.hi + diff.lo);
                // target k 2^-t |A||B| (za's own rounding widened by k 2^-50), plus the summation
                // error of z, plus the rounding of C itself (2^-52 |C|)
                const double tol = fabs(I->alpha) * za[r][c] *
                                       (I->tol_scale * (1.0 + kd * 0x1p-50) + (34.0 + kd / 32.0) * 0x1p-52) +
                                   0x1p-52 * fabs(cv) + 1e-300;
                bad |= !(err <= tol);
            }
        }
    }
    if (bad) atomicOr(fail + I->tile, 1);
}

// ---------------------------------------------------------------- Freivalds probe
// x_vj = +-2^-f_j: the sign from the item's seed, f_j the frexp exponent of op(B)'s column maximum
// (0 for a zero or non-finite column: nothing to test there)
__device__ __forceinline__ double freivalds_x(const FreivaldsItem* I, int v, int64_t j) {
    const unsigned long long b = I->maxb[j];
    if (b == 0 || b >= 0x7FF0000000000000ull) return 0.0;
    const int f = frexp_exp_bits(b);
    const double mag = ldexp(1.0, -f);
    const uint64_t h = mix64(I->seed ^ (static_cast<uint64_t>(v) << 40) ^ static_cast<uint64_t>(j));
    return (h & 1) ? -mag : mag;
}
// acc + x for a double x (exact error term kept)
__device__ __forceinline__ dd dd_add_d(dd acc, double x) {
    dd s = two_sum(acc.hi, x);
    s.lo += acc.lo;
    return two_sum(s.hi, s.lo);
}

// pass 1: thread (p, v) of the block's kFreivaldsP inner indices: u_v,p = sum_j op(B)(p, j) x_vj in
// double-double (each product exact) and ub_v,p = sum_j |op(B)(p, j)| |x_vj|
__global__ void __launch_bounds__(kFreivaldsP * kFreivaldsVecs) freivalds_bx_kernel(
    const FreivaldsItem* __restrict__ items, int count) {
    constexpr int JC = 32, V = kFreivaldsVecs, P = kFreivaldsP;
    const FreivaldsItem* I = items + find_block_item(items, count, blockIdx.x);
    const int64_t p0 = (static_cast<int64_t>(blockIdx.x) - I->block0) * P;
    const int64_t k = I->k, nt = I->nt;
    const int tp = threadIdx.x % P, v = threadIdx.x / P;
    __shared__ double bs[JC][P + 1];
    __shared__ double xs[V][JC];
    dd u{0.0, 0.0};
    double ub = 0.0;
    for (int64_t j0 = 0; j0 < nt; j0 += JC) {
        if (threadIdx.x < V * JC) {
            const int vv = threadIdx.x / JC, jj = threadIdx.x % JC;
            xs[vv][jj] = j0 + jj < nt ? freivalds_x(I, vv, j0 + jj) : 0.0;
        }
        for (int e = threadIdx.x; e < JC * P; e += blockDim.x) {
            int jj, pp;
            if (I->b_rowc) {  // op(B)(p, j) at B[j + p ldb]: j contiguous
                jj = e % JC;
                pp = e / JC;
            } else {          // B[p + j ldb]: p contiguous
                pp = e % P;
                jj = e / P;
            }
            const int64_t p = p0 + pp, j = j0 + jj;
            double b = 0.0;
            if (p < k && j < nt) b = I->b_rowc ? I->B[j + p * I->ldb] : I->B[p + j * I->ldb];
            bs[jj][pp] = b;
        }
        __syncthreads();
#pragma unroll 8
        for (int jj = 0; jj < JC; ++jj) {
            const double b = bs[jj][tp], x = xs[v][jj];
            u = dd_add_d(u, b * x);  // a power-of-two scaling: exact unless it underflows
            ub = fma(fabs(b), fabs(x), ub);
        }
        __syncthreads();
    }
    const int64_t p = p0 + tp;
    if (p < k) {
        I->work[(3 * v + 0) * k + p] = u.hi;
        I->work[(3 * v + 1) * k + p] = u.lo;
        I->work[(3 * v + 2) * k + p] = ub;
    }
}

// pass 2: one thread per tile row i: z_v = alpha (op(A) u_v)_i and y_v = (C x_v)_i in double-double,
// zb_v = (|op(A)| ub_v)_i and yb_v = (|C| |x_v|)_i in FP64; the row fails when |z_v - y_v| exceeds
// |alpha| k 2^-t zb_v (the target summed over the row with weights |x_vj|) widened by the FP64
// rounding of zb (k + nt + 8 terms), plus one rounding of C (2^-52 yb_v), plus the probe's own
// double-double errors (below 2^-90 of the magnitudes), plus the underflow floor
__global__ void __launch_bounds__(kFreivaldsRows) freivalds_check_kernel(const FreivaldsItem* __restrict__ items,
                                                                         int count, int* __restrict__ fail) {
    constexpr int V = kFreivaldsVecs, PC = 256;
    const FreivaldsItem* I = items + find_block_item(items, count, blockIdx.x);
    const int64_t i = (static_cast<int64_t>(blockIdx.x) - I->block0) * kFreivaldsRows + threadIdx.x;
    const int64_t k = I->k, nt = I->nt, mt = I->mt;
    const bool live = i < mt;
    __shared__ double us[V][3][PC];
    dd z[V], y[V];
    double zb[V], yb[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        z[v] = y[v] = dd{0.0, 0.0};
        zb[v] = yb[v] = 0.0;
    }
    for (int64_t p0 = 0; p0 < k; p0 += PC) {
        const int pn = static_cast<int>(min(static_cast<int64_t>(PC), k - p0));
        for (int e = threadIdx.x; e < V * 3 * PC; e += blockDim.x) {
            const int q = e % PC, w = e / PC;  // w = 3 v + component
            us[w / 3][w % 3][q] = q < pn ? I->work[w * k + p0 + q] : 0.0;
        }
        __syncthreads();
        if (live) {
            for (int q = 0; q < pn; ++q) {
                const int64_t p = p0 + q;
                const double a = I->a_rowc ? __ldg(I->A + i + p * I->lda) : __ldg(I->A + p + i * I->lda);
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    z[v] = dd_add_prod(z[v], a, us[v][0][q]);
                    z[v].lo = fma(a, us[v][1][q], z[v].lo);
                    zb[v] = fma(fabs(a), us[v][2][q], zb[v]);
                }
            }
        }
        __syncthreads();
    }
    __shared__ double xs[V][PC];
    for (int64_t j0 = 0; j0 < nt; j0 += PC) {
        const int jn = static_cast<int>(min(static_cast<int64_t>(PC), nt - j0));
        for (int e = threadIdx.x; e < V * PC; e += blockDim.x) {
            const int q = e % PC, v = e / PC;
            xs[v][q] = q < jn ? freivalds_x(I, v, j0 + q) : 0.0;
        }
        __syncthreads();
        if (live) {
            for (int q = 0; q < jn; ++q) {
                const double c = I->C[i + (j0 + q) * I->ldc];
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    y[v] = dd_add_d(y[v], c * xs[v][q]);
                    yb[v] = fma(fabs(c), fabs(xs[v][q]), yb[v]);
                }
            }
        }
        __syncthreads();
    }
    if (!live) return;
    const double al = I->alpha, kd = static_cast<double>(k) + static_cast<double>(nt) + 8.0;
    bool bad = false;
#pragma unroll
    for (int v = 0; v < V; ++v) {
        // alpha z as a double-double: two-product of the high part, the low part rounded once
        const double zh = al * z[v].hi;
        const dd az = two_sum(zh, fma(al, z[v].hi, -zh) + al * z[v].lo);
        const dd diff = dd_add(az, dd{-y[v].hi, -y[v].lo});
        const double err = fabs(diff.hi + diff.lo);
        const double mag = fabs(al) * zb[v];
        const double tol = mag * I->tol_scale * (1.0 + kd * 0x1p-50) + 0x1p-52 * yb[v] + 0x1p-90 * (mag + yb[v]) +
                           1e-300;
        bad |= !(err <= tol);
    }
    if (bad) atomicOr(fail + I->tile, 1);
}

// ---------------------------------------------------------------- double-double reference
// C_hi + C_lo ~= op(A) op(B) and |op(A)| |op(B)| for an m x n block, N/N column-major inputs.
__global__ void __launch_bounds__(256) dd_gemm_nn_kernel(int64_t m, int64_t n, int64_t k, const double* __restrict__ A,
                                                         int64_t lda, const double* __restrict__ B, int64_t ldb,
                                                         double* __restrict__ hi, double* __restrict__ lo,
                                                         double* __restrict__ absab) {
    __shared__ double As[32][33];
    __shared__ double Bs[32][33];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;  // 16 x 16 threads, 2 x 2 outputs each
    const int64_t i0 = static_cast<int64_t>(blockIdx.x) * 32, j0 = static_cast<int64_t>(blockIdx.y) * 32;
    dd acc[2][2] = {{{0, 0}, {0, 0}}, {{0, 0}, {0, 0}}};
    double ab[2][2] = {{0, 0}, {0, 0}};
    for (int64_t p0 = 0; p0 < k; p0 += 32) {
        for (int e = threadIdx.x; e < 32 * 32; e += 256) {
            const int r = e & 31, c = e >> 5;
            As[r][c] = (i0 + r < m && p0 + c < k) ? A[(i0 + r) + (p0 + c) * lda] : 0.0;
            Bs[r][c] = (p0 + r < k && j0 + c < n) ? B[(p0 + r) + (j0 + c) * ldb] : 0.0;
        }
        __syncthreads();
        for (int q = 0; q < 32; ++q)
            for (int a = 0; a < 2; ++a)
                for (int b = 0; b < 2; ++b) {
                    const double x = As[ty + 16 * a][q], y = Bs[q][tx + 16 * b];
                    acc[a][b] = dd_add_prod(acc[a][b], x, y);
                    ab[a][b] = fma(fabs(x), fabs(y), ab[a][b]);
                }
        __syncthreads();
    }
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
            const int64_t i = i0 + ty + 16 * a, j = j0 + tx + 16 * b;
            if (i < m && j < n) {
                hi[i + j * m] = acc[a][b].hi;
                lo[i + j * m] = acc[a][b].lo;
                absab[i + j * m] = ab[a][b];
            }
        }
}

// max over entries of |(C - hi) - lo| / (scale * absab), as float bits for atomicMax
__global__ void error_ratio_kernel(int64_t m, int64_t n, const double* __restrict__ C, int64_t ldc,
                                   const double* __restrict__ hi, const double* __restrict__ lo,
                                   const double* __restrict__ absab, double scale, unsigned int* __restrict__ out) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= m * n) return;
    const int64_t i = e % m, j = e / m;
    const double err = fabs((C[i + j * ldc] - hi[e]) - lo[e]);
    const double t = scale * absab[e];
    float r;
    if (err == 0.0) r = 0.0f;
    else if (!(t > 0.0)) r = __int_as_float(0x7F800000);  // error where none is allowed
    else r = static_cast<float>(err / t);
    if (!(r == r)) r = __int_as_float(0x7F800000);
    atomicMax(out, __float_as_uint(r));  // non-negative floats order like their bits
}

// accuracy of C against the double-double product, as the reference's accuracy bench defines it
// (benchmarks/bench_accuracy.cpp:69-94): the largest |C - (hi + lo)| in units of the spacing above
// |hi| (the smallest subnormal where hi = 0), and how many entries equal RN(hi + lo)
__global__ void accuracy_kernel(int64_t m, int64_t n, const double* __restrict__ C, int64_t ldc,
                                const double* __restrict__ hi, const double* __restrict__ lo,
                                unsigned int* __restrict__ max_ulp, unsigned long long* __restrict__ correct) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    float u = 0.0f;
    bool cr = false;
    if (e < m * n) {
        const int64_t i = e % m, j = e / m;
        const double c = C[i + j * ldc], h = hi[e], l = lo[e];
        const double rn = h + l;  // hi + lo is normalised: their sum rounds the exact value once
        cr = c == rn || (c != c && rn != rn);
        int ex;
        frexp(h, &ex);
        const double ulp = h == 0.0 ? 0x1p-1074 : ldexp(1.0, max(ex - 53, -1074));
        const double err = fabs((c - h) - l) / ulp;
        u = err == err ? static_cast<float>(err) : __int_as_float(0x7F800000);
    }
    for (int o = 16; o > 0; o >>= 1) u = fmaxf(u, __shfl_xor_sync(0xFFFFFFFFu, u, o));
    const unsigned int votes = __popc(__ballot_sync(0xFFFFFFFFu, cr));
    if ((threadIdx.x & 31) == 0) {
        atomicMax(max_ulp, __float_as_uint(u));
        if (votes) atomicAdd(correct, static_cast<unsigned long long>(votes));
    }
}

}  // namespace

void launch_accuracy(int64_t m, int64_t n, const double* C, int64_t ldc, const double* hi, const double* lo,
                     unsigned int* max_ulp, unsigned long long* correct, cudaStream_t st) {
    const int64_t total = m * n;
    accuracy_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, st>>>(m, n, C, ldc, hi, lo, max_ulp, correct);
}

int64_t stat_item_blocks(StatItem& it, int64_t block0) {
    it.block0 = block0;
    if (it.rows <= 0 || it.k <= 0) {
        it.rblocks = 1;
        it.kchunk = 1;
        return 0;
    }
    it.rblocks = it.row_contig ? (it.rows + 31) / 32 : (it.rows + 7) / 8;
    const int64_t chunks = (it.k + 2047) / 2048;
    it.kchunk = (it.k + chunks - 1) / chunks;
    return it.rblocks * chunks;
}

int64_t scale_stat_item_blocks(StatItem& it, int64_t block0) {
    it.block0 = block0;
    it.kchunk = it.k;
    it.rblocks = it.rows <= 0 || it.k <= 0 ? 0 : (it.row_contig ? (it.rows + 31) / 32 : (it.rows + 7) / 8);
    return it.rblocks;
}

void launch_scale_stats(const StatItem* d, const StatItem* h, int count, int64_t blocks, cudaStream_t st) {
    if (count <= 0 || blocks <= 0) return;
    if (h[0].row_contig) scale_stats_kernel<true><<<static_cast<unsigned>(blocks), 256, 0, st>>>(d, count);
    else scale_stats_kernel<false><<<static_cast<unsigned>(blocks), 256, 0, st>>>(d, count);
}

void launch_panel_stats(const StatItem* d, const StatItem* h, int count, int64_t blocks, cudaStream_t st) {
    if (count <= 0 || blocks <= 0) return;
    if (h[0].row_contig) panel_stats_kernel<true><<<static_cast<unsigned>(blocks), 256, 0, st>>>(d, count);
    else panel_stats_kernel<false><<<static_cast<unsigned>(blocks), 256, 0, st>>>(d, count);
}

void launch_tile_features(const FeatureItem* d, int count, float* feat, int* s_analytic, cudaStream_t st) {
    if (count <= 0) return;
    tile_features_kernel<<<(count + 127) / 128, 128, 0, st>>>(d, count, feat, s_analytic);
}

int64_t probe_item_blocks(ProbeItem& it, int64_t block0) {
    it.block0 = block0;
    return (it.mt + kProbeRows - 1) / kProbeRows;
}

void launch_probe(const ProbeItem* d, int count, int64_t blocks, int* fail, cudaStream_t st) {
    if (count <= 0 || blocks <= 0) return;
    probe_kernel<<<static_cast<unsigned>(blocks), kProbeThreads, 0, st>>>(d, count, fail);
}

int64_t freivalds_blocks_pass1(FreivaldsItem& it, int64_t block0) {
    it.block0 = block0;
    return (it.k + kFreivaldsP - 1) / kFreivaldsP;
}
int64_t freivalds_blocks_pass2(FreivaldsItem& it, int64_t block0) {
    it.block0 = block0;
    return (it.mt + kFreivaldsRows - 1) / kFreivaldsRows;
}
void launch_freivalds(const FreivaldsItem* d1, int64_t blocks1, const FreivaldsItem* d2, int64_t blocks2, int count,
                      int* fail, cudaStream_t st) {
    if (count <= 0 || blocks1 <= 0 || blocks2 <= 0) return;
    freivalds_bx_kernel<<<static_cast<unsigned>(blocks1), kFreivaldsP * kFreivaldsVecs, 0, st>>>(d1, count);
    freivalds_check_kernel<<<static_cast<unsigned>(blocks2), kFreivaldsRows, 0, st>>>(d2, count, fail);
}

void launch_dd_gemm_nn(int64_t m, int64_t n, int64_t k, const double* A, int64_t lda, const double* B, int64_t ldb,
                       double* hi, double* lo, double* absab, cudaStream_t st) {
    dim3 grid(static_cast<unsigned>((m + 31) / 32), static_cast<unsigned>((n + 31) / 32));
    dd_gemm_nn_kernel<<<grid, 256, 0, st>>>(m, n, k, A, lda, B, ldb, hi, lo, absab);
}

void launch_error_ratio(int64_t m, int64_t n, const double* C, int64_t ldc, const double* hi, const double* lo,
                        const double* absab, double scale, unsigned int* out, cudaStream_t st) {
    const int64_t total = m * n;
    error_ratio_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, st>>>(m, n, C, ldc, hi, lo, absab, scale,
                                                                                 out);
}

}  // namespace oz2
