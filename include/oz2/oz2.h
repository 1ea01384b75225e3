/*
 * oz2.h - C ABI of the B200-native Ozaki Scheme II FP64 GEMM emulator (liboz2.so).
 *
 * Plain pointers and sizes only. Stream and event arguments are cudaStream_t / cudaEvent_t
 * passed as void*. Matrices are column-major device pointers, as in BLAS. Every entry point
 * returns an oz2_status; oz2_last_error() gives the message of the last failure on a handle.
 *
 * Each entry point replaces one member of the reference's C++ class oz2::Ozaki2
 * (MacraMacra/OS2-Xe, src/ozaki2_gpu.hpp); the citation is given beside it. The C++ header
 * oz2/ozaki2.hpp wraps these functions in a class with the reference's names and exceptions.
 */
#ifndef OZ2_OZ2_H
#define OZ2_OZ2_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oz2_context* oz2_handle;

typedef enum {
    OZ2_OK = 0,
    OZ2_EINVAL = 1,     /* std::invalid_argument in the reference */
    OZ2_ENOMEM = 2,     /* workspace does not fit (std::runtime_error in the reference) */
    OZ2_EINTERNAL = 3,  /* std::runtime_error / std::logic_error */
    OZ2_ETIMEOUT = 4,   /* a device-side wait ran out; no counterpart in the reference */
    OZ2_EOVERFLOW = 5,  /* std::overflow_error */
    OZ2_ECUDA = 6       /* a CUDA runtime call failed */
} oz2_status;

/* Ozaki2(sycl::queue&) / ~Ozaki2(): src/ozaki2_gpu.hpp:680-687.
 * Binds to a caller-owned CUDA stream (NULL = legacy default stream) of the current device. */
int oz2_create(void* stream, oz2_handle* out);
int oz2_destroy(oz2_handle h);
/* rebinds the handle to another stream of the same device (no counterpart: SYCL binds once) */
int oz2_set_stream(oz2_handle h, void* stream);

/* Ozaki2::gemm: src/ozaki2_gpu.hpp:739-760.
 * C = alpha op(A) op(B) + beta C with op in {'N','T','C'} ('C' equals 'T' for real data),
 * num_moduli in [2, 24]. deps: cudaEvent_t[ndeps] the stream waits on first (may be NULL);
 * done: a cudaEvent_t recorded after the last kernel (may be NULL). Asynchronous. */
int oz2_dgemm(oz2_handle h, char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A,
              int64_t lda, const double* B, int64_t ldb, double beta, double* C, int64_t ldc, int num_moduli,
              void* const* deps, int ndeps, void* done);

/* Ozaki2::zgemm: src/ozaki2_gpu.hpp:764-786. Complex data interleaved (re, im) as
 * std::complex<double>; alpha and beta point to {re, im} on the HOST. 3M form, 3s INT8 GEMMs. */
int oz2_zgemm(oz2_handle h, char ta, char tb, int64_t m, int64_t n, int64_t k, const double* alpha,
              const double* A, int64_t lda, const double* B, int64_t ldb, const double* beta, double* C,
              int64_t ldc, int num_moduli, void* const* deps, int ndeps, void* done);

/* One problem of a grouped call: C = alpha op(A) op(B) + beta C (real). */
typedef struct {
    char ta, tb;     /* 'N', 'T' or 'C' */
    int num_moduli;  /* s in [2, 24], per problem */
    int64_t m, n, k;
    double alpha, beta;
    const double* A;
    int64_t lda;
    const double* B;
    int64_t ldb;
    double* C;
    int64_t ldc;
} oz2_dgemm_problem;

/* Many independent emulated DGEMMs of uneven m, n, k, ops and s in one set of launches: one
 * grouped scale and split per kernel variant, one persistent tcgen05 GEMM over every
 * (problem, modulus, tile) job, one CRT per distinct s. No counterpart in the reference
 * (equivalent to `count` calls of Ozaki2::gemm, src/ozaki2_gpu.hpp:739-760, with the same
 * results bit for bit). A problem whose num_moduli is OZ2_S_ADAPTIVE (-1) instead takes the
 * adaptive s per tile of oz2_dgemm_adaptive (mode 0, DGEMM-level target of 53 bits): those
 * problems run together after the fixed-s ones, and the call then does not run in graph mode
 * (OZ2_EINVAL), since the adaptive choice reads tile statistics back to the host. Arguments are
 * checked for every problem before anything runs; C blocks must not overlap. */
#define OZ2_S_ADAPTIVE (-1)
int oz2_dgemm_grouped(oz2_handle h, int count, const oz2_dgemm_problem* problems, void* const* deps, int ndeps,
                      void* done);
/* Grouped calls are captured in a CUDA graph on first use and replayed when the same problem
 * list (shapes, pointers, scalars) comes again; the workspace must not grow in between. */
int oz2_set_graph_mode(oz2_handle h, int enable);
/* kernels launched through this handle since oz2_create, a CUDA-graph replay counting its kernel
 * nodes (no counterpart in the reference) */
int oz2_kernel_launches(oz2_handle h, int64_t* out);
/* GEMM kernel configuration: tile width along the rows of C (bn = 128 or 256), raster group of
 * column tiles (group_j), persistent CTAs (ctas, 0 = one per SM); bn = 0 returns to the
 * autotuned / heuristic choice. get returns the configuration of the last call. */
int oz2_set_gemm_config(oz2_handle h, int bn, int group_j, int ctas);
int oz2_get_gemm_config(oz2_handle h, int* out3);
/* Times the candidate configurations on these problems (C is overwritten), remembers the
 * fastest for problem lists of the same shapes and returns it in out3 (may be NULL). */
int oz2_autotune_grouped(oz2_handle h, int count, const oz2_dgemm_problem* problems, int* out3);

/* Adaptive number of moduli per C tile (no counterpart in the reference). Target: every entry
 * within k 2^-target_bits (|A||B|)_ij of the exact product, the classical error bound of a native
 * FP64 GEMM for target_bits = 53 ("DGEMM-level error"). Per tile of tile x tile entries (default
 * 512), s comes from
 *   mode 0: the MLP (oz2_mlp_set_weights; a tile takes the largest class over itself and its
 *           up to 8 neighbours in the problem), capped by the arbiter's s, for problems with
 *           beta = 0 and tiles without a certificate (the others take the arbiter's s); tiles below
 *           the arbiter's s are probed (C x against A (B x) with x = e_j for 8 columns j, each entry
 *           checked) and rerun at it when the probe fails; without weights it behaves as mode 4
 *   mode 1: the analytic s of the tile: smallest s whose tk >= R + 2 + t - floor(log2(k - 1)),
 *           R the largest exponent gap below the row / column maximum in the tile's panels
 *   mode 2: the analytic s of the whole problem (the largest over its tiles)
 *   mode 3: each problem's own num_moduli, 2..32 (tiled like the other modes)
 *   mode 4: the arbiter's s of the tile (no MLP, no probe: every tile meets the target)
 *   mode 5: the arbiter's s of the whole problem (the largest over its tiles)
 * The arbiter of a tile is the smaller of its analytic s and, for problems with a tile whose analytic
 * s is 23 or more (k <= 65472), its certified s: the smallest s for which a rigorous entrywise
 * bound of the emulation's error (row / column sums of |A| and |B| against a bf16 lower bound of
 * |A||B| from a tcgen05 GEMM) meets the target in every entry of the tile. In modes 0 and 4 a
 * problem runs as one task at the largest s of its tiles (or in native FP64) when that costs no
 * more than its tiles as chosen, counting a tile task 12 % dearer and native FP64 as 63 moduli.
 * Above s = 24 the adaptive path uses moduli sets of its own (s = 25..32: pairwise-coprime
 * integers <= 256 taken greedily from the top; up to 124 bits per element), so a tile whose
 * arbiter needs more than the 91 bits of 24 moduli still runs emulated; the MLP's last class means
 * "more than 24" and answers 25. In modes 0-2, 4 and 5 a tile that no s <= 32 brings to the
 * target runs as a native FP64 GEMM (cuBLAS DGEMM), the whole problem in one call when all its
 * tiles do; the analytic rule sends a tile there when a gap reaches 63 binades (its histogram's
 * last bin).
 * stats (may be NULL, 10 entries): tiles, sum of s over emulated tiles (reruns included), probed
 * tiles, rerun tiles, sum of s of the reruns (33 for native), sum of the arbiter's s (33 for native),
 * MLP used, int8 multiply-adds of the emulated tiles (s m_t n_t k summed, reruns included),
 * native tiles, native FP64 multiply-adds. The host waits in the middle of the call for the tile
 * statistics (and in mode 0 for the probe). Those reads, and the uploads of item tables, are copy
 * kernels on an internal highest-priority stream, not copy-engine transfers, so host-device copies
 * that the caller queues on other streams do not delay the call. With profiling on,
 * oz2_stage_times reports scale (with the tile statistics, features and MLP), split, GEMM and CRT
 * summed over the tile batches; the probe and native tiles are in none of them. */
int oz2_dgemm_adaptive(oz2_handle h, int count, const oz2_dgemm_problem* problems, int target_bits, int mode,
                       int64_t* stats);
/* tile edge (multiple of 128) and the MLP decision threshold: s is the smallest class whose
 * cumulative predicted probability reaches it */
int oz2_set_adaptive_options(oz2_handle h, int tile, float threshold);
/* the probe of mode 0 (no counterpart in the reference): 0 (default) checks kProbeCols = 8
 * stratified random columns of each probed tile entry by entry against A B summed in FP64; 1 is the
 * Freivalds test, C x against alpha A (B x) in double-double for two random vectors x with
 * x_j = +-2^-f_j (f_j the exponent of op(B)'s column maximum), row by row against alpha k 2^-t
 * (|A| (|B| |x|))_i; 2 runs both (a tile fails when either fails); 3 runs none, so the MLP's s
 * stands unchecked (for measuring what the probes catch). A tile that meets the target passes
 * every kind; a failing tile is rerun at its arbiter's s. */
int oz2_set_probe_kind(oz2_handle h, int kind);
/* with profiling on: device time of the last oz2_dgemm_adaptive's probe and of its native FP64
 * tiles (out2 = {probe_ms, native_ms}) */
int oz2_adaptive_stage_times(oz2_handle h, double* out2);
/* algorithmic bytes of the last oz2_dgemm_adaptive's INT8 GEMMs (no counterpart in the reference):
 * out3 = {plane bytes read (each split panel once), residue bytes written, tile batches (one GEMM
 * launch each)}; the yardstick for the GEMM's measured DRAM traffic */
int oz2_adaptive_gemm_bytes(oz2_handle h, int64_t* out3);
/* out4 = {parameters, features, classes (s = 2..24 and one for more than 24), hidden width} of the MLP */
int oz2_mlp_info(int* out4);
/* loads the MLP parameters (host floats); NULL unloads */
int oz2_mlp_set_weights(oz2_handle h, const float* params, int nparams);
/* trains in place (host params) on device features [count][features] and labels (s values);
 * loss (host, epochs floats, may be NULL) receives the mean loss per epoch */
int oz2_mlp_train(oz2_handle h, int count, const float* d_features, const int* d_labels, int epochs, float lr,
                  unsigned int seed, float* params, float* loss);
/* s per sample (device) and class probabilities (device, may be NULL) for host params */
int oz2_mlp_infer(oz2_handle h, const float* params, int count, const float* d_features, float threshold, int* d_s,
                  float* d_probs);
/* features [tiles][features] and analytic s per tile (device outputs, tiles in problem order,
 * column tiles outer, row tiles inner); ntiles receives the count */
int oz2_tile_features(oz2_handle h, int count, const oz2_dgemm_problem* problems, int target_bits,
                      float* d_features, int* d_s_analytic, int64_t* ntiles);
/* double-double product hi + lo ~= A B and |A| |B| (m x n, leading dimension m) of column-major
 * A (m x k) and B (k x n) on the device: the reference the labels are measured against */
int oz2_dd_reference(oz2_handle h, int64_t m, int64_t n, int64_t k, const double* A, int64_t lda, const double* B,
                     int64_t ldb, double* hi, double* lo, double* absab);
/* max_ulp = max over entries of |C - (hi + lo)| in units of the spacing above |hi|;
 * correctly_rounded = entries equal to RN(hi + lo) (hi, lo from oz2_dd_reference, m x n,
 * leading dimension m); synchronises. No counterpart in the reference's API (its accuracy bench
 * reports the same two figures, benchmarks/bench_accuracy.cpp:69-94). */
int oz2_accuracy(oz2_handle h, int64_t m, int64_t n, const double* C, int64_t ldc, const double* hi,
                 const double* lo, double* max_ulp, int64_t* correctly_rounded);
/* out = max over entries of |C - (hi + lo)| / (k 2^-target_bits |A||B|); synchronises */
int oz2_error_ratio(oz2_handle h, int64_t m, int64_t n, int64_t k, const double* C, int64_t ldc, const double* hi,
                    const double* lo, const double* absab, int target_bits, float* out);

/* The reference's Ozaki Scheme I comparison baseline, oz1::Ozaki1::gemm (benchmarks/ozaki1_gpu.hpp:85-147):
 * C = A B for column-major, untransposed A (m x k) and B (k x n) with L in [2, 9] digits of 7 bits
 * (7L - 2 bits per element, L (L + 1) / 2 INT8 GEMMs), the same results as the reference bit for bit.
 * k * 4096 must stay below 2^31. Asynchronous on the handle's stream. */
int oz2_ozaki1_dgemm(oz2_handle h, int64_t m, int64_t n, int64_t k, const double* A, int64_t lda, const double* B,
                     int64_t ldb, double* C, int64_t ldc, int L);

/* Ozaki2::precision_bits / precision_bits_complex / moduli_for_bits: src/ozaki2_gpu.hpp:689-700, :762 */
int oz2_precision_bits(int64_t k, int num_moduli, int* out);
int oz2_precision_bits_complex(int64_t k, int num_moduli, int* out);
int oz2_moduli_for_bits(int64_t k, int bits, int* out);

/* Ozaki2::set_workspace_limit / set_resident_hint / release_workspace: src/ozaki2_gpu.hpp:702-710 */
int oz2_set_workspace_limit(oz2_handle h, size_t bytes);
int oz2_set_resident_hint(oz2_handle h, size_t bytes);
int oz2_release_workspace(oz2_handle h);

/* Ozaki2::stage_times: src/ozaki2_gpu.hpp:716-737. out = {scale_ms, split_ms, gemm_ms, crt_ms}.
 * Zeros unless profiling is on (the reference's queue property enable_profiling). Waits for
 * the last call. */
int oz2_set_profiling(oz2_handle h, int enable);
int oz2_stage_times(oz2_handle h, double* out4);

/* Ozaki2::last_tiling: src/ozaki2_gpu.hpp:712, TileInfo :47-53.
 * out = {mb, nb, pm, pn, k_chunks, workspace_bytes} */
int oz2_last_tiling(oz2_handle h, int64_t* out6);

/* Ozaki2::set_tuning: src/ozaki2_gpu.hpp:713, Tuning :41-45. The reference's three knobs are
 * Xe2-specific. pow2_tiles keeps its meaning: with it set (the default) the tiling of C under a
 * workspace limit considers power-of-two tile edges first. batched_gemm and pad_lda are accepted
 * and stored but change nothing here: every INT8 GEMM of a call is one persistent launch, and the
 * planes are always written in a padded, pre-tiled layout. */
int oz2_set_tuning(oz2_handle h, int batched_gemm, int pad_lda, int pow2_tiles);

/* Device-side error word: non-zero after a kernel's bounded wait ran out (OZ2_ETIMEOUT).
 * Synchronises the handle's stream, returns and clears the word. */
int oz2_check_device_error(oz2_handle h);

/* Test of the failure path (no counterpart in the reference; process-wide, read at each GEMM
 * launch, so set it only while no other call is being made). wait_limit_ns bounds every
 * mbarrier wait of the INT8 GEMM (0 restores the 2 s default); with stall_mma != 0 the GEMM's
 * MMA issuer issues nothing, so the copy and epilogue waits run out: the kernel records a code in
 * the error word, drains its copies, frees its tensor memory and returns, the call's C is not
 * valid, and oz2_check_device_error (oz2_noalloc_check_device_error for oz2_dgemm_noalloc)
 * returns OZ2_ETIMEOUT. Calls after oz2_set_failure_test(0, 0) compute normally. */
int oz2_set_failure_test(int64_t wait_limit_ns, int stall_mma);

/* Kernel of the real split (no counterpart in the reference; process-wide, read when a call
 * builds its launches, so set it only while no other call is being made): 0 (default) the
 * integer-pipe (dp4a) split; 1 the tensor-core split, which computes the byte dot products of
 * every residue with one tcgen05 u8 x u8 MMA per 512 elements (measured slower on B200: it is
 * bound by per-element instruction overhead, not by the dot products). Both write identical
 * planes. Complex operands always use the integer-pipe split. OZ2_EINVAL for other values. */
int oz2_set_split_kernel(int kind);

/* Kernel of the real CRT (no counterpart in the reference; process-wide, read when a call builds
 * its launches): 0 the dp2a kernel; 1 the tensor-core CRT, whose limb sums are one tcgen05 u8 x
 * u8 MMA per 128 entries; 2 (default) the tensor-core CRT for plans of 7 and 8 limbs (s = 26..32),
 * the dp2a kernel below. All produce identical C. Complex operands always use the dp2a kernel. OZ2_EINVAL
 * for other values. */
int oz2_set_crt_kernel(int kind);

/* Scale pass fused into the split (no counterpart in the reference, which runs them as two passes
 * over A and B; process-wide, read when a call builds its launches): with on != 0 a real operand
 * of oz2_dgemm / oz2_dgemm_grouped whose k is at most 2048 (1024 when its plane rows are contiguous
 * in memory: op(A) = A, op(B) = B^T) is scaled and split by one kernel that owns whole rows, takes
 * their maxima and splits them while they are still in L2. Results are identical. Default off: on
 * B200 it measured neutral on one DGEMM and 2.7 % slower on a group of 512 small DGEMMs. */
int oz2_set_scale_fusion(int on);

/* CRT in the GEMM's epilogue (no counterpart in the reference; process-wide, read when a call
 * builds its launches): with on != 0 real problems of oz2_dgemm / oz2_dgemm_grouped with s <= 8
 * and k <= 65408 run one GEMM launch per plan whose epilogue keeps each 128 x 128 tile's residues
 * of all s moduli in tensor memory and reconstructs C there: no residue planes in HBM and no CRT
 * launch. Results are identical. Default off: on B200 it measured slower than the GEMM followed by
 * the CRT launch (the reconstruction runs on the GEMM's eight epilogue warps). */
int oz2_set_crt_fusion(int on);

/* Emulated DGEMM for callers that cannot allocate device memory. No counterpart in the
 * reference. Same arguments, checks and results as oz2_dgemm, but no handle: it works on the
 * given stream and the current device and allocates nothing. Its scratch is a 64 MiB static
 * device array of the library (held by every GPU that loads it until the process exits), so
 * problems needing more scratch are rejected with OZ2_EINVAL (m = n = k = 1024 at 16 moduli
 * fits). The first call on each device looks the array up and should come before any stream
 * capture. All calls share the array: calls that overlap on the GPU race. */
int oz2_dgemm_noalloc(void* stream, char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha,
                      const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
                      int64_t ldc, int num_moduli);
/* The device error word of oz2_dgemm_noalloc (no counterpart in the reference): synchronises the
 * stream, returns OZ2_ETIMEOUT (and clears the word) when a bounded wait of the last call's GEMM
 * ran out, so its C is not valid; the next oz2_dgemm_noalloc clears the word as well, so check
 * before it. Allocates nothing. Neither entry point may be used after cudaDeviceReset: the array's
 * device address is looked up once per device. */
int oz2_noalloc_check_device_error(void* stream);

/* message of the last failed call on the handle (or of the last failed handle-less call) */
const char* oz2_last_error(oz2_handle h);
const char* oz2_status_string(int status);

#ifdef __cplusplus
}
#endif
#endif
