// oz2_certify.cu - a rigorous number of moduli per C tile from the data (no counterpart in the
// reference, whose s is fixed per call).
//
// With D_i = tk - e_i and E_j = tk - f_j (e_i, f_j the frexp exponents of the row / column
// maxima), the emulation computes sum_p x_ip y_pj exactly, x_ip = RNE(a_ip 2^D_i) = a_ip 2^D_i +
// alpha_ip and y_pj = b_pj 2^E_j + beta_pj with |alpha|, |beta| <= 1/2, then rounds (once, and
// once more for alpha != 1). The scaled error sum_p (x beta + alpha y - alpha beta) is at most
// 1/2 sum |x| + 1/2 sum |y| + k/4 <= 1/2 2^D_i R_i + 1/2 2^E_j S_j + 3k/4, so
//   |C_ij - (AB)_ij| <= 1/2 2^(f_j - tk) R_i + 1/2 2^(e_i - tk) S_j + 3k/4 2^(e_i + f_j - 2 tk)
//                       + two roundings of 2^-53 |C_ij|,
// R_i = sum_p |a_ip| and S_j = sum_p |b_pj|. With R'_i = R_i 2^-e_i, S'_j = S_j 2^-f_j and
// G_ij <= (|A||B|)_ij 2^-(e_i + f_j) a lower bound, the target |C - AB| <= k 2^-t (|A||B|)_ij
// (t = 53: DGEMM-level) holds at tk when, with B = k - 2^(t - 52) (the two roundings, each at
// most 2^-53 |C|, take 2^(t - 52) of the k units of 2^-t (|A||B|)_ij), for every entry,
//   1/2 2^-tk (R'_i + S'_j) <= (1 - 2^-10) B 2^-t c G_ij   and
//   3k/4 2^-2tk            <= 2^-10 B 2^-t c G_ij,
// c = 1 - 2^-6 absorbing the bf16 rounding of the GEMM inputs (2^-9 each), its FP32
// accumulation (k 2^-24 for k <= 2^16), the FP64 sums R', S' and the FP32 ratio below. The
// largest tk that this asks over the tile's entries gives the certified s: the smallest s whose
// plan reaches it. Entries of an all-zero row of A or column of B are exact at any s and are
// skipped; G_ij = 0 elsewhere (products that all underflowed) asks for native FP64.
//
// G comes from the persistent tcgen05 GEMM (kind::f16, bf16 operands, FP32 accumulators in TMEM)
// over bf16 planes of the scaled magnitudes that cert_prep_kernel writes; the GEMM's epilogue
// keeps only the two maxima per tile, and cert_tile_kernel turns them into s.
#include <cuda_bf16.h>

#include <cmath>

#include "oz2_adaptive.cuh"
#include "oz2_kernels.cuh"

namespace oz2 {
namespace {

__device__ __forceinline__ int frexp_exp_bits(unsigned long long b) {  // frexp exponent of |x| from bits
    const int be = static_cast<int>((b >> 52) & 0x7FF);
    return be ? be - 1022 : -1010 - __clzll(static_cast<long long>(b));
}
__device__ __forceinline__ double pow2(int k) {  // 2^k, k in [-1022, 1023]
    return __longlong_as_double(static_cast<long long>(k + 1023) << 52);
}
__device__ __forceinline__ uint32_t bf16x2(double lo, double hi) {
    return static_cast<uint32_t>(__bfloat16_as_ushort(__double2bfloat16(lo))) |
           (static_cast<uint32_t>(__bfloat16_as_ushort(__double2bfloat16(hi))) << 16);
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

// scaled magnitude |x| 2^-e as two exact power-of-two products (e in [-1073, 1024])
struct Scale {
    double s1, s2;
    bool live;
};
__device__ __forceinline__ Scale row_scale(unsigned long long mb) {
    Scale sc{1.0, 1.0, mb != 0 && mb < 0x7FF0000000000000ull};
    if (sc.live) {
        const int e = frexp_exp_bits(mb), e1 = (-e) / 2;
        sc.s1 = pow2(e1);
        sc.s2 = pow2(-e - e1);
    }
    return sc;
}

// the 16 bytes of plane row r that hold elements 8c .. 8c + 7 (c counts 8-element chunks over
// the padded k): tile (r / 128, c / 8), row r % 128, chunk c % 8 swizzled by r % 8
__device__ __forceinline__ uint4* chunk_ptr(uint8_t* planes, int64_t kb_total, int64_t r, int64_t c) {
    const int rr = static_cast<int>(r & 127), cc = static_cast<int>(c & 7);
    return reinterpret_cast<uint4*>(planes + ((r >> 7) * kb_total + (c >> 3)) * kTileBytes + rr * kTileK +
                                    ((cc ^ (rr & 7)) << 4));
}

// Rows contiguous: 32 rows (lanes) x 8 slices of the chunk range (warps) per block; each thread
// sums its slice in k order, the 8 slice sums are added in slice order (a fixed order: the sums
// are the same on every run). k contiguous: one warp per row, lane l takes chunks l, l + 32, ...,
// then a fixed shuffle tree. Every chunk is eight loads in flight and one 16-byte store.
template <bool ROWC>
__global__ void __launch_bounds__(256) cert_prep_kernel(const CertPrepItem* __restrict__ items, int count) {
    const CertPrepItem* I = items + find_block_item(items, count, blockIdx.x);
    const int64_t local = static_cast<int64_t>(blockIdx.x) - I->block0;
    const int64_t k = I->k, ldx = I->ldx, rows = I->rows, kb_total = I->kb_total;
    const int64_t nchunk = kb_total * 8;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    auto chunk = [&](int64_t r, int64_t c, const Scale& sc, const double* x, int64_t step, double& sum) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int64_t p = 8 * c + u;
            v[u] = sc.live && p < k ? (fabs(__ldg(x + p * step)) * sc.s1) * sc.s2 : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) sum += v[u];
        *chunk_ptr(I->planes, kb_total, r, c) =
            make_uint4(bf16x2(v[0], v[1]), bf16x2(v[2], v[3]), bf16x2(v[4], v[5]), bf16x2(v[6], v[7]));
    };
    if (ROWC) {
        __shared__ double part[8][32];
        const int64_t r = local * kCertRowsPerBlock + lane;  // < rows_pad: padding rows write zeros
        double sum = 0.0;
        if (r < I->rows_pad) {
            const Scale sc = r < rows ? row_scale(I->maxbits[r]) : Scale{1.0, 1.0, false};
            const int64_t per = (nchunk + 7) / 8, c0 = warp * per, c1 = min(nchunk, c0 + per);
            const double* x = I->X + r;
            for (int64_t c = c0; c < c1; c += 2) {  // two chunks' sixteen loads in flight
                double v[16];
#pragma unroll
                for (int u = 0; u < 16; ++u) {
                    const int64_t p = 8 * c + u;
                    v[u] = sc.live && p < k && c + u / 8 < c1 ? (fabs(__ldg(x + p * ldx)) * sc.s1) * sc.s2 : 0.0;
                }
#pragma unroll
                for (int h2 = 0; h2 < 2; ++h2) {
                    if (c + h2 >= c1) break;
                    const double* w = v + 8 * h2;
#pragma unroll
                    for (int u = 0; u < 8; ++u) sum += w[u];
                    *chunk_ptr(I->planes, kb_total, r, c + h2) = make_uint4(
                        bf16x2(w[0], w[1]), bf16x2(w[2], w[3]), bf16x2(w[4], w[5]), bf16x2(w[6], w[7]));
                }
            }
        }
        part[warp][lane] = sum;
        __syncthreads();
        if (warp == 0 && r < rows) {
            double t = 0.0;
#pragma unroll
            for (int w = 0; w < 8; ++w) t += part[w][lane];
            I->rsum[r] = t;
        }
    } else {
        const int64_t r = local * 8 + warp;
        if (r >= I->rows_pad) return;
        const Scale sc = r < rows ? row_scale(I->maxbits[r]) : Scale{1.0, 1.0, false};
        double sum = 0.0;
        for (int64_t c = lane; c < nchunk; c += 32) chunk(r, c, sc, I->X + r * ldx, 1, sum);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
        if (lane == 0 && r < rows) I->rsum[r] = sum;
    }
}

// One warp per tile: the lanes scan the tile's row and column maxima for a non-finite one
// (kNativeS then: those rows' outputs are NaN at any s and the analytic rule decides), lane 0
// turns the GEMM's two maxima into the certified s.
__global__ void __launch_bounds__(128) cert_tile_kernel(const CertTileItem* __restrict__ items, int count) {
    const int t = blockIdx.x * 4 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (t >= count) return;
    const CertTileItem* I = items + t;
    bool bad = false;
    for (int64_t i = lane; i < I->mb; i += 32) bad |= I->maxa[i] >= 0x7FF0000000000000ull;
    for (int64_t j = lane; j < I->nb; j += 32) bad |= I->maxb[j] >= 0x7FF0000000000000ull;
    const bool nonfinite = __any_sync(0xFFFFFFFFu, bad);
    if (lane != 0) return;
    const float q1 = __uint_as_float(I->q[0]), q2 = __uint_as_float(I->q[1]);
    int s = kNativeS;
    const double k = static_cast<double>(I->k), tb = static_cast<double>(I->target_bits);
    const double B = k - exp2(tb - 52.0);
    if (!nonfinite && B > 0.0 && q1 < INFINITY && q2 < INFINITY) {
        if (q1 == 0.0f) {
            s = 2;  // every entry is exact: all rows of A or all columns of B are zero
        } else {
            // the FP32 ratios carry a relative error below 2^-21: widened by 2^-20
            const double c = 1.0 - 0x1p-6;
            const double l1 = log2(static_cast<double>(q1) * (1.0 + 0x1p-20)) + tb - 1.0 - log2(B * c * (1.0 - 0x1p-10));
            const double l2 = 0.5 * (log2(static_cast<double>(q2) * (1.0 + 0x1p-20)) + tb + 10.0 - log2(B / k * c));
            const double need = ceil(fmax(l1, l2) + 1e-9);
            for (int q = 2; q <= kMaxModuliExt; ++q)
                if (I->tk[q] > 0 && static_cast<double>(I->tk[q]) >= need) {
                    s = q;
                    break;
                }
        }
    }
    *I->s_out = s;
}

}  // namespace

int64_t cert_prep_blocks(CertPrepItem& it, int64_t block0) {
    it.block0 = block0;
    it.blocks = it.row_contig ? (it.rows_pad + kCertRowsPerBlock - 1) / kCertRowsPerBlock : (it.rows_pad + 7) / 8;
    return it.blocks;
}

void launch_cert_prep(const CertPrepItem* d, const CertPrepItem* h, int count, int64_t blocks, cudaStream_t st) {
    if (count <= 0 || blocks <= 0) return;
    if (h[0].row_contig) cert_prep_kernel<true><<<static_cast<unsigned>(blocks), 256, 0, st>>>(d, count);
    else cert_prep_kernel<false><<<static_cast<unsigned>(blocks), 256, 0, st>>>(d, count);
}

void launch_cert_tiles(const CertTileItem* d, int count, cudaStream_t st) {
    if (count <= 0) return;
    cert_tile_kernel<<<static_cast<unsigned>((count + 3) / 4), 128, 0, st>>>(d, count);
}

}  // namespace oz2
