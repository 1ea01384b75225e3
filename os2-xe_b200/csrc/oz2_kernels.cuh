// oz2_kernels.cuh - parameter blocks and launchers of the Ozaki-II device phases:
//   scale : row / column max |x| of op(A), op(B) as raw FP64 bits       (oz2_split.cu)
//   split : exact power-of-two scaling + symmetric INT8 residues, written
//           as pre-tiled 128x128-byte swizzled planes                   (oz2_split.cu)
//   gemm  : tcgen05 kind::i8 products with the mod-m reduction fused
//           into the epilogue, uint8 residue planes out                  (oz2_gemm.cu)
//   crt   : CRT reconstruction + unscaling + alpha/beta update           (oz2_crt.cu)
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
// GEMM tile: 128 columns j of C (MMA M, TMEM lanes) x 256 rows i of C (MMA N, TMEM columns)
constexpr int kGemmJ = 128;
constexpr int kGemmI = 256;
// k blocks per exact int32 accumulation: 1023 * 128 = 130944 <= 131071, so that
// k_chunk * 128^2 < 2^31 (ref src/ozaki2_gpu.hpp:32)
constexpr int kChunkKB = 1023;

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline int64_t round_up(int64_t a, int64_t b) { return ceil_div(a, b) * b; }

// One operand side of the scale and split phases, in terms of the plane rows r (rows of op(A)
// for A, columns of op(B) for B) and the inner index p < k.
struct SideDesc {
    const double* X;   // first element of row 0 (already offset for tiles)
    int64_t ldx;       // leading dimension in elements (complex: in complex elements)
    int64_t rows;      // valid plane rows
    int64_t k;
    bool row_contig;   // element (r, p) at X[r + p*ldx]; else at X[p + r*ldx]
    bool cplx;         // interleaved (re, im)
    bool conj;         // use conj(x) (complex only)
};

// plane geometry of one side
struct PlaneGeom {
    int64_t rows_pad;    // rows padded to the tile multiple this side needs (128 for j, 256 for i)
    int64_t kb_total;    // k blocks per row block
    int64_t plane_bytes; // bytes of one plane
};
inline PlaneGeom plane_geom(int64_t rows, int64_t k, int row_multiple) {
    PlaneGeom g;
    g.rows_pad = round_up(rows > 0 ? rows : 1, row_multiple);
    g.kb_total = ceil_div(k, kTileK);
    g.plane_bytes = g.rows_pad * g.kb_total * kTileK;
    return g;
}

void launch_scale(const SideDesc& sd, unsigned long long* maxbits, int num_sms, cudaStream_t st);

// planes: s planes (3s for complex: groups re | im | re+im, group stride s * plane_bytes)
void launch_split(const SideDesc& sd, const unsigned long long* maxbits, int tk, const ModConst* mc, int s,
                  int8_t* planes, const PlaneGeom& g, cudaStream_t st);

struct GemmArgs {
    const int8_t* planes_i;   // I side (op(A) rows), plane rows padded to 256
    const int8_t* planes_j;   // J side (op(B) columns), plane rows padded to 128
    uint8_t* resid;           // residue planes: [g][t][j * ldr + i]
    int64_t pstride_i, pstride_j;  // bytes per plane
    int64_t rstride;               // bytes per residue plane
    int64_t ldr;                   // residue plane leading dimension, multiple of 32
    int64_t m, n;                  // valid i rows, j rows
    int64_t kb_total;              // k blocks per row block (same on both sides)
    int64_t kb0, kb1;              // k-block range of this launch
    int s, groups;
    int accumulate;                // add to the residues already in resid (k chunks after the first)
    const ModConst* mc;            // host array of s constants (copied into the kernel parameters)
    int* err;                      // device error word
};
void launch_gemm(const GemmArgs& a, int num_sms, cudaStream_t st);

struct CrtArgs {
    const uint8_t* resid;
    int64_t rstride, ldr;
    int64_t m, n;                  // tile dims
    const unsigned long long* maxA;  // row max bits of op(A) for the tile rows
    const unsigned long long* maxB;  // column max bits of op(B) for the tile columns
    int tk;
    bool cplx;
    double alpha[2], beta[2];
    double* C;                     // tile origin (complex: interleaved)
    int64_t ldc;
    const Plan* plan;
};
void launch_crt(const CrtArgs& a, cudaStream_t st);

// C = beta * C (beta == 0 writes zeros), the k == 0 / alpha == 0 path
void launch_scale_c(double* C, int64_t ldc, int64_t m, int64_t n, const double* beta, bool cplx, cudaStream_t st);

}  // namespace oz2
