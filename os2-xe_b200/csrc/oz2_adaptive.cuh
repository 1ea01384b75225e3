// oz2_adaptive.cuh - item tables and launchers of the adaptive-s subsystem (tile statistics,
// features, analytic s, the Freivalds-style probe, the double-double reference used to label
// training tiles) and of the small MLP that predicts s per tile. No counterpart in the
// reference, whose number of moduli is fixed per call.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "oz2_plan.hpp"

namespace oz2 {

constexpr int kGapBins = 64;     // exponent gaps 0..63 (63 = "63 or more"), plus a zero counter
constexpr int kFeatures = 18;
constexpr int kHidden = 32;
// s = 2..32 run emulated (s = 25..32 with the extended moduli sets); kNativeS marks a tile that no
// s <= 32 brings to the target, run as a native FP64 GEMM
constexpr int kNativeS = kMaxModuliExt + 1;
// the MLP's classes: s = 2..24 and one for "more than 24" (s = 25 as its answer: a lower bound
// that the probe checks, or the arbiter's s where a certificate takes the tile)
constexpr int kClasses = kMaxModuli;
// per-call statistics of oz2_dgemm_adaptive
constexpr int kAdaptiveStats = 10;
constexpr int kMlpParams = kHidden * kFeatures + kHidden + kHidden * kHidden + kHidden + kClasses * kHidden + kClasses;
constexpr int kProbeCols = 8;    // columns per probed tile, each entry checked on its own
constexpr int kProbeChunk = 512;  // inner-index chunk of the probe's B columns in shared memory
constexpr int kProbeThreads = 128;
constexpr int kProbeRowsPerThread = 2;
constexpr int kProbeRows = kProbeThreads * kProbeRowsPerThread;  // tile rows per probe block

// histogram of exponent gaps for the rows [0, rows) of one panel (rows of op(A) or columns of
// op(B)), all k; layout like ScaleItem
struct StatItem {
    const double* X;
    int64_t ldx, rows, k;
    int row_contig;
    unsigned long long* maxbits;        // row maxima of the panel rows (written by scale_stats)
    unsigned int* hist;                 // kGapBins + 1 counters, zeroed before the launch
    int64_t kchunk, block0, rblocks;
};

// one C tile: its two panels' histograms and maxima, k, target, tk per s for this k
struct FeatureItem {
    const unsigned int* hist_a;
    const unsigned int* hist_b;
    const unsigned long long* maxbits_a;
    const unsigned long long* maxbits_b;
    int64_t rows_a, rows_b, k;
    int target_bits;
    int tk[kMaxModuliExt + 1];  // tk[s] for s = 2..32 (0 where s is too small for k)
};

// probe of one computed tile (pointers at the tile's first row / column)
struct ProbeItem {
    const double* A;  // op(A) rows of the tile
    const double* B;  // op(B) columns of the tile
    const double* C;
    int64_t lda, ldb, ldc, mt, nt, k;
    int a_rowc;       // op(A)(i, p) at A[i + p lda] (else A[p + i lda])
    int b_rowc;       // op(B)(p, j) at B[j + p ldb] (else B[p + j ldb])
    double alpha, tol_scale;  // tol_scale = k 2^-t
    uint64_t seed;
    int tile;         // index into the failure flags
    int64_t block0;
};

// Freivalds probe of one computed tile (C x against alpha A (B x) in double-double):
// kFreivaldsVecs random vectors x_v with x_vj = +-2^-f_j (f_j the frexp exponent of op(B)'s
// column maximum, 0 for a zero or non-finite column), so every product with x is exact. Pass 1
// (one block per kFreivaldsP inner indices): u_v = op(B) x_v in double-double and ub_v = |op(B)||x_v|.
// Pass 2 (one block per kFreivaldsRows tile rows): per row i, |alpha (op(A) u_v)_i - (C x_v)_i| <=
// alpha k 2^-t (|op(A)| ub_v)_i widened for the probe's own roundings. A tile that meets the
// target entry by entry always passes; the test sees an error entry only through its row sum.
constexpr int kFreivaldsVecs = 2;
constexpr int kFreivaldsP = 64;     // inner indices per pass-1 block
constexpr int kFreivaldsRows = 128;  // tile rows per pass-2 block (one per thread)
struct FreivaldsItem {
    const double* A;  // op(A) rows of the tile
    const double* B;  // op(B) columns of the tile
    const double* C;
    const unsigned long long* maxb;  // column maxima (raw bits) of op(B) for the tile's columns
    double* work;     // 3 kFreivaldsVecs k doubles: u_v hi, u_v lo, ub_v
    int64_t lda, ldb, ldc, mt, nt, k;
    int a_rowc, b_rowc;
    double alpha, tol_scale;  // tol_scale = k 2^-t
    uint64_t seed;
    int tile;
    int64_t block0;
};
int64_t freivalds_blocks_pass1(FreivaldsItem& it, int64_t block0);
int64_t freivalds_blocks_pass2(FreivaldsItem& it, int64_t block0);
void launch_freivalds(const FreivaldsItem* d1, int64_t blocks1, const FreivaldsItem* d2, int64_t blocks2, int count,
                      int* fail, cudaStream_t st);

// ---- certified s (a rigorous entrywise a-priori bound, see oz2_certify.cu)
// one panel side of a problem: the scaled magnitudes |x| 2^-e_r of its rows (rows of op(A) or
// columns of op(B)) as bf16 planes in the GEMM's tiled layout (128 x 128-byte swizzled tiles,
// 64 elements per 128-byte row, padding rows and k zero), and their sums R'_r in FP64
struct CertPrepItem {
    const double* X;
    int64_t ldx, rows, k;
    int row_contig;                     // rows contiguous (X[r + p ldx]) or k contiguous (X[p + r ldx])
    const unsigned long long* maxbits;  // row maxima (raw bits) of the rows
    uint8_t* planes;
    int64_t rows_pad, kb_total;         // plane geometry (kb_total 128-byte blocks of 64 elements)
    double* rsum;                       // R'_r (0 for a zero or non-finite row)
    int64_t block0, blocks;
};
// one C tile: the two maxima the certificate GEMM left for it, its rows' and columns' maxima
struct CertTileItem {
    const unsigned int* q;  // FP32 bits: max (R'_i + S'_j) / G_ij, max 1 / G_ij (0 when all exact)
    const unsigned long long* maxa;
    const unsigned long long* maxb;
    int64_t mb, nb, k;
    int target_bits;
    int tk[kMaxModuliExt + 1];
    int* s_out;  // smallest certified s, kNativeS where none is (or the tile has a non-finite row)
};
constexpr int kCertRowsPerBlock = 32;   // rows-contiguous prep: 32 rows x 8 k slices per block
constexpr int64_t kCertMaxK = 65472;     // one k chunk of the GEMM (1023 blocks of 64 bf16)
int64_t cert_prep_blocks(CertPrepItem& it, int64_t block0);
void launch_cert_prep(const CertPrepItem* d, const CertPrepItem* h, int count, int64_t blocks, cudaStream_t st);
void launch_cert_tiles(const CertTileItem* d, int count, cudaStream_t st);

int64_t stat_item_blocks(StatItem& it, int64_t block0);
void launch_panel_stats(const StatItem* d, const StatItem* h, int count, int64_t blocks, cudaStream_t st);
// the scale pass and the panel statistics in one launch: a block owns whole rows, takes their
// maxima (written to maxbits) and then reads the same rows again, from the L2, for the gap
// histogram; for problems with k up to kFusedStatsMaxK (a row then stays well inside the L2)
constexpr int64_t kFusedStatsMaxK = 16384;
int64_t scale_stat_item_blocks(StatItem& it, int64_t block0);
void launch_scale_stats(const StatItem* d, const StatItem* h, int count, int64_t blocks, cudaStream_t st);
void launch_tile_features(const FeatureItem* d, int count, float* feat, int* s_analytic, cudaStream_t st);
int64_t probe_item_blocks(ProbeItem& it, int64_t block0);
void launch_probe(const ProbeItem* d, int count, int64_t blocks, int* fail, cudaStream_t st);
void launch_dd_gemm_nn(int64_t m, int64_t n, int64_t k, const double* A, int64_t lda, const double* B, int64_t ldb,
                       double* hi, double* lo, double* absab, cudaStream_t st);
void launch_error_ratio(int64_t m, int64_t n, const double* C, int64_t ldc, const double* hi, const double* lo,
                        const double* absab, double scale, unsigned int* out, cudaStream_t st);
// max error in ulps of RN(hi + lo) (float bits) and the count of entries equal to RN(hi + lo)
void launch_accuracy(int64_t m, int64_t n, const double* C, int64_t ldc, const double* hi, const double* lo,
                     unsigned int* max_ulp, unsigned long long* correct, cudaStream_t st);

// MLP: kFeatures -> kHidden (ReLU) -> kHidden (ReLU) -> kClasses, parameters packed as
// W1[kHidden][kFeatures] b1 W2[kHidden][kHidden] b2 W3[kClasses][kHidden] b3.
// s = 2 + the smallest class whose cumulative softmax probability reaches `threshold`.
void launch_mlp_infer(const float* params, int count, const float* feat, float threshold, int* s_out,
                      float* probs_out, cudaStream_t st);
// mini-batch Adam with cross-entropy, one block; loss_out[epoch] = mean training loss
void launch_mlp_train(float* params, int count, const float* feat, const int* label, int epochs, float lr,
                      unsigned int seed, float* loss_out, cudaStream_t st);

}  // namespace oz2
