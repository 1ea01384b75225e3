// oz2_kernels.cuh - descriptor tables and launchers of the Ozaki-II device phases:
//   scale : row / column max |x| of op(A), op(B) as raw FP64 bits       (oz2_split.cu)
//   split : exact power-of-two scaling + symmetric INT8 residues, written
//           as pre-tiled 128x128-byte swizzled planes                   (oz2_split.cu)
//   gemm  : tcgen05 kind::i8 products with the mod-m reduction fused
//           into the epilogue, uint8 residue planes out                  (oz2_gemm.cu)
//   crt   : CRT reconstruction + unscaling + alpha/beta update           (oz2_crt.cu)
// Every phase works on a table of items in device memory, so that one launch serves one
// problem or a whole group of independent problems; blocks (or persistent jobs) are mapped to
// items through per-item prefix offsets.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "oz2_plan.hpp"

namespace oz2 {

// ---- plane layout shared by split (writer) and gemm (reader)
// A plane holds one modulus (and one 3M group) of one operand: rows x k int8 values stored as
// row blocks of 128 rows, each made of k blocks of 128 bytes; one 128x128 tile is 16 KiB, row
// r of the tile at r*128, 16-byte chunk c of that row at chunk position c ^ (r % 8). Rows and
// k are zero-padded to whole tiles.
constexpr int kTileRows = 128;
constexpr int kTileK = 128;
constexpr int kTileBytes = kTileRows * kTileK;
// GEMM tile: 128 columns j of C (MMA M, TMEM lanes) x BN rows i of C (MMA N, TMEM columns),
// BN in {128, 256}. I-side planes are padded to 256 rows so both widths can read them.
constexpr int kGemmJ = 128;
constexpr int kGemmIPad = 256;
// k blocks per exact int32 accumulation: 1023 * 128 = 130944 <= 131071, so that
// k_chunk * 128^2 < 2^31 (ref src/ozaki2_gpu.hpp:32)
constexpr int kChunkKB = 1023;

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

inline int64_t round_up(int64_t a, int64_t b) { return ceil_div(a, b) * b; }

// plane geometry of one side
struct PlaneGeom {
    int64_t rows_pad;     // rows padded to the tile multiple this side needs
    int64_t kb_total;     // k blocks per row block
    int64_t plane_bytes;  // bytes of one plane
};
inline PlaneGeom plane_geom(int64_t rows, int64_t k, int row_multiple) {
    PlaneGeom g;
    g.rows_pad = round_up(rows > 0 ? rows : 1, row_multiple);
    g.kb_total = ceil_div(k, kTileK);
    g.plane_bytes = g.rows_pad * g.kb_total * kTileK;
    return g;
}

// ---- scale: one item per operand side of a problem. Plane rows r are rows of op(A) (A side)
// or columns of op(B) (B side); p < k is the inner index.
struct ScaleItem {
    const double* X;
    int64_t ldx, rows, k;
    int row_contig;  // element (r, p) at X[r + p*ldx]; else at X[p + r*ldx] (complex: pairs)
    int cplx;
    unsigned long long* out;  // rows entries, zeroed before the launch
    int64_t kchunk;           // inner indices per block
    int64_t block0;           // first block of this item in the launch
    int64_t rblocks;          // row blocks (blocks = rblocks * k chunks)
};

// ---- split: one item per operand panel
struct SplitItem {
    const double* X;
    int64_t ldx, rows, k;
    int row_contig, cplx, conj;
    int tk, s;
    const unsigned long long* maxbits;  // of the panel's rows (written by the fused scale + split)
    int8_t* planes;                     // s planes (complex: 3 groups of s)
    int64_t plane_bytes, kb_total, rows_pad;
    int64_t block0, rblocks, kblocks;   // blocks = rblocks * kblocks
    ModConst mc[kMaxModuliExt];
    // tc: the tensor-core split runs this item (real operands); block0 is then its first unit of
    // 512 elements (4 rows x 128 inner indices, or 16 x 32 when rows are contiguous), rblocks x
    // kblocks its units
    int tc;
    // fuse: the scale pass is fused into this item's split (real operands, k <= kFuseMaxK): the
    // kernel takes the row maxima itself and writes them to maxbits; rblocks blocks of whole rows
    int fuse;
};
// largest k for which the scale pass is fused into the split (k contiguous / rows contiguous)
constexpr int64_t kFuseMaxK = 2048;
constexpr int64_t kFuseMaxKRowc = 1024;

// ---- gemm: one item per problem; jobs = groups * s * tiles, each job runs all k chunks
constexpr int kMaxOz1Pairs = 45;  // Ozaki Scheme I: L (L + 1) / 2 digit pairs, L <= 9

struct GemmItem {
    const int8_t* planes_i;  // I side (op(A) rows), plane rows padded to 256
    const int8_t* planes_j;  // J side (op(B) columns), plane rows padded to 128
    uint8_t* resid;          // residue planes [g][t]; entry (i, j) at (i / 32) * 32 n + j * 32 + i % 32
    int64_t pstride_i, pstride_j, rstride, ldr, m, n, kb_total;
    int64_t tiles, job0;
    int tiles_i, tiles_j, s, groups;
    uint32_t mod_m[kMaxModuliExt], mod_mu[kMaxModuliExt], mod_kbias[kMaxModuliExt];
    uint32_t mod_kbias30[kMaxModuliExt], mod_mx31[kMaxModuliExt];  // exact quotient, kb_total <= kExactKB
    uint32_t mod_mxs[kMaxModuliExt];                                // its shift (oz2_plan.hpp)
    // Ozaki-I mode only: job index t is the digit pair (pair_a[t], pair_b[t]) on anti-diagonal
    // pair_d[t]; the int32 products are added into acc[d][i acc_ld + j] (int64)
    int64_t* acc;
    int64_t acc_ld, acc_plane;
    uint8_t pair_a[kMaxOz1Pairs], pair_b[kMaxOz1Pairs], pair_d[kMaxOz1Pairs];
    // certificate mode only: bf16 planes (64 elements per 128-byte row), the scaled sums R' of
    // op(A)'s rows and S' of op(B)'s columns, and per adaptive tile (cert_tile rows and columns,
    // cert_na tiles down a column of tiles) two FP32 maxima as bits: (R'_i + S'_j) / G_ij, 1 / G_ij
    const double* cert_ra;
    const double* cert_sb;
    unsigned int* cert_q;
    int64_t cert_tile, cert_na;
    // CRT in the epilogue (launch_gemm_crt): C (rows i, columns j of this item) and its alpha /
    // beta update, the maxima of op(A)'s rows and op(B)'s columns for the unscaling
    double* C;
    int64_t ldc;
    const unsigned long long* crt_maxA;
    const unsigned long long* crt_maxB;
    int crt_tk;
    double crt_alpha, crt_beta;
};
// largest s whose residues fit in tensor memory beside the two accumulators (BN = 128: 8 x 32
// columns of packed bytes), so that the GEMM's epilogue can run the CRT itself
constexpr int kCrtFusedMaxS = 8;

// ---- crt: one item per problem; all items of a launch share s
struct CrtItem {
    const uint8_t* resid;
    int64_t rstride, gstride, ldr, m, n, ldc;
    const unsigned long long* maxA;  // row max bits of op(A) for the problem rows
    const unsigned long long* maxB;  // column max bits of op(B) for the problem columns
    int tk;
    double ar, ai, br, bi;
    double* C;
    int64_t block0, iblocks;  // blocks = ceil(n / jb) * iblocks
    int tq, jb;               // a block: tq threads (4 rows each) along i x jb columns, tq * jb = 256
    // mma: the tensor-core CRT (real items, crt_uses_mma): block0 is the first super-tile of 32
    // rows x 16 columns (four tcgen05 MMAs of 128 entries) and iblocks the super-tiles along i;
    // otherwise the dp2a kernel's geometry
    int mma;
};

// host-side helpers filling the launch-geometry fields; they return the blocks of the item
int64_t scale_item_blocks(ScaleItem& it, int num_sms, int64_t block0);
int64_t split_item_blocks(SplitItem& it, int64_t block0);
// the split's geometry for the kernel that will run the item: the tensor-core split for real
// items while it is selected, else split_item_blocks; sets it.tc
int64_t split_geometry(SplitItem& it, int64_t block0);
// process-wide selection of the real split: 0 the dp4a kernel (default), 1 the tensor-core split
void set_split_path(int tc);
int split_path();
// process-wide: whether real operands with k <= kFuseMaxK (kFuseMaxKRowc when rows are contiguous)
// take the fused scale + split (default off: measured neutral on one DGEMM and 2.7 % slower on a
// group of 512 small DGEMMs, where the separate passes spread over more blocks); fuse_scale tells
// whether an operand qualifies
void set_scale_fusion(int on);
bool fuse_scale(bool cplx, bool row_contig, int64_t k);
int64_t crt_item_blocks(CrtItem& it, int64_t block0);

// launches over device tables (d_items) whose host copies (h_items) give the geometry
void launch_scale(const ScaleItem* d_items, const ScaleItem* h_items, int count, int64_t blocks, cudaStream_t st);
// all items of one split launch share row_contig, cplx, tc and the narrow/wide/widest limb path;
// err: the device error word for the tensor-core split's bounded wait on its MMA (may be null
// only for launches without tc items)
void launch_split(const SplitItem* d_items, const SplitItem* h_items, int count, int64_t blocks, int* err,
                  cudaStream_t st);

struct GemmConfig {
    int bn = 256;        // tile width along i (MMA N): 256 or 128
    int group_j = 16;    // raster: column tiles that share a row panel in flight
    int ctas = 0;        // persistent CTAs (0 = one per SM)
};
void launch_gemm(const GemmItem* d_items, int count, int64_t jobs, const GemmConfig& cfg, int num_sms, int* err,
                 cudaStream_t st);
// the same GEMM on bf16 planes of scaled magnitudes, with the certificate's maxima in the
// epilogue instead of residues (one job per tile; items as for launch_gemm with s = 1)
void launch_gemm_cert(const GemmItem* d_items, int count, int64_t jobs, int num_sms, int* err, cudaStream_t st);
// the same GEMM with the CRT in its epilogue (real items of one plan with s <= kCrtFusedMaxS and
// at most kExactKB k blocks): one job per 128 x 128 tile runs all s moduli, keeps the residues in
// tensor memory and writes C; no residue planes and no CRT launch. BN is 128.
void launch_gemm_crt(const GemmItem* d_items, int count, int64_t jobs, const Plan& plan, int group_j, int num_sms,
                     int* err, cudaStream_t st);
// process-wide: whether fixed-s real problems that qualify take launch_gemm_crt (default off:
// measured slower than the GEMM followed by the CRT launch, since the reconstruction of a tile's
// 16384 entries runs on the GEMM's eight epilogue warps while the MMA pipeline waits)
void set_crt_fusion(int on);
int crt_fusion();
// the same GEMM for the Ozaki Scheme I baseline: digit-pair jobs, int64 atomic sums per diagonal
void launch_gemm_oz1(const GemmItem* d_items, int count, int64_t jobs, const GemmConfig& cfg, int num_sms, int* err,
                     cudaStream_t st);
// Ozaki Scheme I digits: item.s = L balanced base-128 digits of RNE(x 2^e), e = tk - frexp_exp(max)
void launch_slice(const SplitItem* d_items, const SplitItem* h_items, int count, int64_t blocks, cudaStream_t st);
// Ozaki Scheme I: C = 2^(7 (L - 1) - D_i - E_j) * Horner_d(acc[d]) in double-double, NaN for
// non-finite rows / columns
void launch_oz1_horner(const int64_t* acc, int64_t m, int64_t n, int L, const unsigned long long* maxA,
                       const unsigned long long* maxB, int tk, double* C, int64_t ldc, cudaStream_t st);
int64_t gemm_tiles_i(int64_t m, int bn);

// whether launch_crt runs the tensor-core CRT for this plan (real items only): process-wide path
// 0 the dp2a kernel, 1 the tensor-core CRT, 2 (default) the tensor-core CRT from
// kCrtTcMinLimbs limbs on (7 and 8 limbs: s = 26..32, where it measured as fast or faster: B200,
// 4096^2 x 1024, s = 29: 0.56 against 0.67 ms; s = 20: 0.47 against 0.28); the items' `mma` flag
// must match
constexpr int kCrtTcMinLimbs = 7;
bool crt_uses_mma(const Plan& plan, bool cplx);
void set_crt_path(int path);
int crt_path();
// sets the tensor-core CRT kernels' shared-memory attribute (with prepare_gemm_kernels)
cudaError_t prepare_crt_kernels();
// all items of one CRT launch share s (the CRT table is a kernel parameter); err: the device error
// word for the real kernel's bounded wait on its MMA (may be null)
void launch_crt(const CrtItem* d_items, int count, int64_t blocks, const Plan& plan, bool cplx, int* err,
                cudaStream_t st);

// sets the shared-memory attribute of the GEMM and tensor-core split kernels (once per device,
// before any graph capture)
cudaError_t prepare_gemm_kernels();
cudaError_t prepare_split_kernels();
// Failure-path test of the GEMM's bounded waits (process-wide, read at each launch): wait_ns
// limits every mbarrier wait (0 = the 2 s default); with stall set the MMA issuer of every CTA
// issues nothing, so the other roles' waits run out, record their code in the error word, drain
// their copies, free TMEM and return.
void set_gemm_failure_test(uint64_t wait_ns, int stall);

// Copies up to kParamBlobBytes of host data to device memory by passing them as the parameter
// of a one-block kernel: no staging buffer, no memcpy, capturable in a graph.
constexpr size_t kParamBlobBytes = 30 * 1024;
void launch_write_blob(const void* src, size_t bytes, void* dst, cudaStream_t st);

// Copies bytes with SM loads and stores; either side may be pinned host memory, which unified
// addressing maps into the device's address space. A call moves its own small data (item tables
// in, tile decisions out) only through these kernels, in stream order on the SMs: a
// cudaMemcpyAsync on the call's stream waits behind the bulk host copies other streams queued
// on the copy engines.
void launch_sm_copy(const void* src, void* dst, size_t bytes, cudaStream_t st);
// bytes of dst set to `value`, by a kernel
void launch_fill(void* dst, unsigned char value, size_t bytes, cudaStream_t st);

// C = beta * C (beta == 0 writes zeros), the k == 0 / alpha == 0 path
void launch_scale_c(double* C, int64_t ldc, int64_t m, int64_t n, const double* beta, bool cplx, cudaStream_t st);

}  // namespace oz2
