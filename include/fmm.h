/*
 * fmm.h -- C ABI of the B200 fast-matrix-multiplication engine (libfmm.so).
 *
 * Plain pointers and sizes only; no exceptions cross this boundary.  All
 * matrices are column-major doubles (floats for the _f32 entry points and
 * fmm_sgemm), as in the reference's Matrix<Scalar>
 * view (linalg/linalg.hpp:41-192): element (i, j) of a matrix with leading
 * dimension ld is at ptr[i + j * ld].  Unless a function says "host", its
 * matrix pointers are CUDA device pointers on the handle's device.
 *
 * The engine replaces the reference's per-algorithm entry point
 *   template <class Scalar> double <ns>::FastMatmul(Matrix<Scalar>& A,
 *       Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps, double x = 1e-8,
 *       Scalar alpha = 1, Scalar beta = 0)
 * (algorithms/strassen.hpp:661-722 and every other header in algorithms/), the
 * classical MatMul (linalg/linalg.hpp:261-269) and the error metric
 * MaxRelativeDiff (linalg/linalg.hpp:280-295).  include/fmm/algorithms.hpp
 * re-creates the reference's C++ surface on top of these functions.
 */
#ifndef FMM_H_
#define FMM_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum fmm_status {
  FMM_OK = 0,
  FMM_ERR_INVALID_ARGUMENT = 1,
  FMM_ERR_UNKNOWN_ALGORITHM = 2,
  FMM_ERR_OUT_OF_MEMORY = 3,
  FMM_ERR_CUDA = 4,
  FMM_ERR_NOT_SUPPORTED = 5,
  FMM_ERR_WORKSPACE_TOO_SMALL = 6,
  FMM_ERR_TIMEOUT = 7
} fmm_status;

/* Recursion schedules.  The numbering follows the reference's parallel
 * modes _DFS_PAR_=1, _BFS_PAR_=2, _HYBRID_PAR_=3 (util/common.hpp:13-15).
 *   DFS     one sub-problem at a time at every level; the R products of a
 *           deepest-level sub-problem go out as one grouped launch.
 *   BFS     every level is one grouped launch over all its sub-problems
 *           (all R^l operand formations, all R^steps leaf products).
 *   HYBRID  depth-first over the top levels, breadth-first below; the split
 *           is the shallowest one whose workspace fits the limit, with at
 *           least two depth-first levels when num_steps >= 3 (one
 *           depth-first level plans exactly like BFS, since the top level
 *           has a single sub-problem).
 *   AUTO    BFS for num_steps <= 2 (or the shallowest split that fits the
 *           workspace limit), HYBRID for num_steps >= 3, which measured as
 *           fast as BFS or faster there (no result changes: every schedule
 *           gives the same bits). */
typedef enum fmm_schedule {
  FMM_SCHEDULE_AUTO = 0,
  FMM_SCHEDULE_DFS = 1,
  FMM_SCHEDULE_BFS = 2,
  FMM_SCHEDULE_HYBRID = 3
} fmm_schedule;

/* Precision of the leaf products (no counterpart in the reference, which
 * multiplies in the Scalar type of its Matrix).  The operand formations and
 * the M -> C combinations are FP64 in both.
 *   FP64        FP64 tensor-core GEMM (DMMA).
 *   SPLIT_BF16  every leaf operand row (A) / column (B) is scaled by a power
 *               of two and split into `split_slices` BF16 digit slices of 8
 *               bits; the S(S+1)/2 leading slice products run on the BF16
 *               tensor cores (tcgen05) with exact FP32 accumulation over
 *               k groups of 128 (256 for the two leading diagonals at 3
 *               slices or fewer), recombined in FP64.  Error of one leaf
 *               product: |C - AB|_ij <~ 3 * 2^-8S * k * max|A_i.| * max|B_.j|;
 *               S = 5 stays near 1e-14 relative for well-scaled operands.
 *   SPLIT_INT8  the same scaling, split into `split_slices` signed 8-bit
 *               digit slices of 7 bits (|digit| <= 64); the S(S+1)/2 leading
 *               slice products run on the INT8 tensor cores (tcgen05
 *               kind::i8, twice the BF16 rate) with exact int32
 *               accumulation over k groups of up to 32768, recombined in
 *               FP64.  Error of one leaf product:
 *               |C - AB|_ij <~ (S + 2) * 2^-7S * k * max|A_i.| * max|B_.j|;
 *               6 slices are about as accurate as 5 BF16 slices.
 * In both split forms a row of a leaf A or a column of a leaf B that holds an
 * Inf or a NaN makes every entry of that leaf's product it reaches NaN. */
typedef enum fmm_precision {
  FMM_PRECISION_FP64 = 0,
  FMM_PRECISION_SPLIT_BF16 = 1,
  FMM_PRECISION_SPLIT_INT8 = 2
} fmm_precision;

#define FMM_SPLIT_MIN_SLICES 2
#define FMM_SPLIT_MAX_SLICES 6
#define FMM_SPLIT_DEFAULT_SLICES 5
#define FMM_SPLIT_INT8_MAX_SLICES 8
#define FMM_SPLIT_INT8_DEFAULT_SLICES 6

typedef struct fmm_handle_s* fmm_handle;

/* Tile configuration of the FP64 tensor-core GEMM (no counterpart in the
 * reference, whose leaves call the host BLAS).  Both configurations sum every
 * output element over the same k order, so the choice changes speed only,
 * never a result.
 *   AUTO   per launch: SMALL where 128-row tiles would pad the rows of the
 *          launch's problems by more than 7% beyond 64-row tiles, else LARGE
 *          (a batch whose items ask for different ones gets two launches).
 *   LARGE  128 x 64 tiles, two CTAs per SM (the faster one on large products).
 *   SMALL  64 x 64 tiles, three CTAs per SM. */
typedef enum fmm_gemm_tile {
  FMM_GEMM_TILE_AUTO = 0,
  FMM_GEMM_TILE_LARGE = 1,
  FMM_GEMM_TILE_SMALL = 2
} fmm_gemm_tile;

typedef struct fmm_options {
  fmm_schedule schedule;    /* default FMM_SCHEDULE_AUTO */
  fmm_precision precision;  /* default FMM_PRECISION_FP64 */
  int split_slices;         /* slices per operand: SPLIT_BF16 2..6 (0 = default 5), SPLIT_INT8 2..8 (0 = 6) */
  int dfs_levels;           /* HYBRID only: depth-first levels; -1 = choose */
  size_t workspace_limit;   /* bytes; 0 = the handle's limit */
  int gemm_tile;            /* fmm_gemm_tile of the FP64 leaf and fringe products */
} fmm_options;

/* Fills *opts with the defaults above. */
void fmm_options_init(fmm_options* opts);

/* Handles: one per host thread (a handle is not internally locked). */
fmm_status fmm_handle_create(fmm_handle* out, int device);
fmm_status fmm_handle_destroy(fmm_handle h);
/* Stream for all work of the handle (a cudaStream_t; NULL = legacy default). */
fmm_status fmm_set_stream(fmm_handle h, void* stream);
/* Frees the handle's grow-on-demand device buffers (the S/T/M workspace and
 * the staging of the host-pointer and FP32 entry points) once the work
 * queued on its stream is done; the next call allocates again.  The
 * reference's MemoryManager frees its pools when the multiply ends
 * (util/MemoryManager.hpp:26-42); a handle keeps them across calls until
 * this call or fmm_handle_destroy. */
fmm_status fmm_release_workspace(fmm_handle h);
/* Test support, no counterpart in the reference (which has no device
 * workspace): grows the handle's workspace to at least `bytes` and fills all
 * of it with the byte `pattern` (0xFF makes every double a NaN), then
 * synchronises.  A later call that read a temporary before writing it would
 * carry the pattern into C. */
fmm_status fmm_debug_fill_workspace(fmm_handle h, size_t bytes, int pattern);
/* Test support, no counterpart in the reference: in a library built with
 * device-side checks (libfmm_checked.so, -DFMM_DEVICE_CHECKS) the grouped
 * GEMM and the formation and combination kernels check the problems and
 * tiles they decode from their descriptors and that the temporaries they
 * write or read lie inside the running program's workspace; a failed check
 * skips the access and sets a bit here (1: GEMM problem index, 2: GEMM tile
 * origin, 4: formation write, 8: combination read).  Reads the bits of the
 * current device's launches since the last call, clears them, and returns
 * FMM_ERR_NOT_SUPPORTED (flags 0) in the regular library. */
fmm_status fmm_debug_check_flags(unsigned* flags);
/* Upper bound on the workspace the handle may allocate (0 = 60% of the
 * device memory that is free when the handle is created). */
fmm_status fmm_set_workspace_limit(fmm_handle h, size_t bytes);
/* Message for the last failing call on this host thread ("" if none). */
const char* fmm_last_error(void);

/* Algorithm registry: every algorithm the reference generates headers for. */
int fmm_num_algorithms(void);
const char* fmm_algorithm_name(int alg); /* the reference namespace, e.g. "grey424_26_206" */
const char* fmm_algorithm_header(int alg); /* the reference header, e.g. "fast424_26_206.hpp" */
int fmm_algorithm_lookup(const char* name_or_header); /* -1 if unknown */
fmm_status fmm_algorithm_info(int alg, int* m0, int* k0, int* n0, int* rank, int* approximate);

/* C := alpha * A * B + beta * C with `num_steps` recursive levels of
 * algorithm `alg` and parameter x (lambda of approximate algorithms),
 * exactly as <ns>::FastMatmul(A, B, C, num_steps, x, alpha, beta) computes it
 * (algorithms/strassen.hpp:661-722): the same floor sub-blocking, operand
 * additions in the same order and rounding, multipliers folded into the leaf
 * products' alpha, M->C combination with beta at the top level, and dynamic
 * peeling of the fringes at every level (linalg/linalg.hpp:201-244).  As in
 * the reference, num_steps == 0 is one classical product that ignores beta.
 * Device pointers; runs on the handle's stream; returns once the work is
 * queued (the call does not synchronise).  opts may be NULL. */
fmm_status fmm_fast_matmul(fmm_handle h, int alg, const double* A, int64_t lda, const double* B, int64_t ldb,
                           double* C, int64_t ldc, int64_t m, int64_t k, int64_t n, int num_steps, double x,
                           double alpha, double beta, const fmm_options* opts);

/* Same with HOST matrices (pageable or pinned): A, B and (when beta != 0 and
 * num_steps > 0) C are copied to the device, the product runs, C is copied
 * back; the call returns when C is on the host.  *elapsed_ms (may be NULL)
 * receives the wall time of the whole call, copies included. */
fmm_status fmm_fast_matmul_host(fmm_handle h, int alg, const double* A, int64_t lda, const double* B, int64_t ldb,
                                double* C, int64_t ldc, int64_t m, int64_t k, int64_t n, int num_steps, double x,
                                double alpha, double beta, const fmm_options* opts, double* elapsed_ms);
/* Pipelined form of fmm_fast_matmul_host, no counterpart in the reference
 * (whose FastMatmul returns when C is done): queues the copy of A, B (and C
 * when it is read) to the device, the product, and the copy of C back to
 * the host, and returns without waiting.  Two calls may be in flight per
 * handle; each uses one of two device staging slots in turn, so the next
 * call's operands travel to the device and the previous call's C travels
 * back while this call's product runs.  A third call waits, on the device,
 * for the slot's earlier C to have left.  Every host buffer of a queued call
 * must stay valid and unchanged until fmm_host_sync returns, and no queued
 * call may read host memory that another queued call writes (a call that
 * reads C, beta != 0, is ordered after the other slot's copy of C).  Pinned
 * host memory lets the copies overlap the products; pageable memory works
 * but serialises them.  fmm_fast_matmul_host first waits for queued calls. */
fmm_status fmm_fast_matmul_host_async(fmm_handle h, int alg, const double* A, int64_t lda, const double* B,
                                      int64_t ldb, double* C, int64_t ldc, int64_t m, int64_t k, int64_t n,
                                      int num_steps, double x, double alpha, double beta, const fmm_options* opts);
/* Waits until every call queued by fmm_fast_matmul_host_async has put its C
 * on the host; returns the first device-side error of those calls. */
fmm_status fmm_host_sync(fmm_handle h);

/* Device workspace the call above needs (bytes), for the schedule chosen. */
fmm_status fmm_workspace_query(fmm_handle h, int alg, int64_t m, int64_t k, int64_t n, int num_steps,
                               const fmm_options* opts, size_t* bytes);

/* Classical product C := alpha * A * B + beta * C with the engine's own FP64
 * tensor-core GEMM (the leaf kernel); MatMul in linalg/linalg.hpp:261-269
 * with alpha taken from C's multiplier.  beta == 0 does not read C. */
fmm_status fmm_dgemm(fmm_handle h, const double* A, int64_t lda, const double* B, int64_t ldb, double* C,
                     int64_t ldc, int64_t m, int64_t k, int64_t n, double alpha, double beta);

/* Classical product C := alpha * A * B + beta * C computed split-BF16 with
 * `slices` slices (0 = default) on the BF16 tensor cores (no counterpart in
 * the reference).  Device pointers; queued on the handle's stream. */
fmm_status fmm_dgemm_split_bf16(fmm_handle h, const double* A, int64_t lda, const double* B, int64_t ldb,
                                double* C, int64_t ldc, int64_t m, int64_t k, int64_t n, double alpha, double beta,
                                int slices);

/* The same product computed split-INT8 (FMM_PRECISION_SPLIT_INT8) with
 * `slices` slices (0 = default 6) on the INT8 tensor cores. */
fmm_status fmm_dgemm_split_int8(fmm_handle h, const double* A, int64_t lda, const double* B, int64_t ldb,
                                double* C, int64_t ldc, int64_t m, int64_t k, int64_t n, double alpha, double beta,
                                int slices);

/* Same with HOST matrices: A, B (and C when beta != 0) are copied in, the
 * product runs on the engine's GEMM, C is copied back; returns when C is on
 * the host.  MatMul(A, B, C, beta) of linalg/linalg.hpp:261-269 over host
 * buffers, for the C++ adapter (include/fmm/matrix.hpp). */
fmm_status fmm_dgemm_host(fmm_handle h, const double* A, int64_t lda, const double* B, int64_t ldb, double* C,
                          int64_t ldc, int64_t m, int64_t k, int64_t n, double alpha, double beta);

/* FP32 operands: the reference's templates with Scalar = float --
 * <ns>::FastMatmul<float> (algorithms/strassen.hpp:661-722 and the other
 * headers) and MatMul<float>, whose leaf is sgemm (linalg/linalg.hpp:261-269,
 * linalg/blas_wrap.hpp:116-120).  The operands are widened to FP64 once
 * (exact), the product runs on the FP64 engine, and C is rounded to FP32
 * once (round to nearest), so every result is at least as accurate as the
 * reference's, which rounds in FP32 at every addition and leaf product.
 * opts == NULL selects split-INT8 leaf products with FMM_F32_DEFAULT_SLICES
 * slices (34 bits per operand entry, beyond FP32's 24); other options are
 * taken as given (FMM_PRECISION_FP64 runs FP64 leaves, SPLIT_BF16 BF16
 * slices).  Device pointers,
 * the handle's stream; FP64 staging of m*k + k*n + m*n doubles is held by
 * the handle.  num_steps == 0 ignores beta, as FastMatmul does. */
#define FMM_F32_DEFAULT_SLICES 5
fmm_status fmm_fast_matmul_f32(fmm_handle h, int alg, const float* A, int64_t lda, const float* B, int64_t ldb,
                               float* C, int64_t ldc, int64_t m, int64_t k, int64_t n, int num_steps, double x,
                               float alpha, float beta, const fmm_options* opts);
fmm_status fmm_sgemm(fmm_handle h, const float* A, int64_t lda, const float* B, int64_t ldb, float* C, int64_t ldc,
                     int64_t m, int64_t k, int64_t n, float alpha, float beta, const fmm_options* opts);
/* The same with HOST matrices; they return when C is on the host (for the
 * C++ adapter's Matrix<float>). */
fmm_status fmm_fast_matmul_f32_host(fmm_handle h, int alg, const float* A, int64_t lda, const float* B, int64_t ldb,
                                    float* C, int64_t ldc, int64_t m, int64_t k, int64_t n, int num_steps, double x,
                                    float alpha, float beta, const fmm_options* opts, double* elapsed_ms);
fmm_status fmm_sgemm_host(fmm_handle h, const float* A, int64_t lda, const float* B, int64_t ldb, float* C,
                          int64_t ldc, int64_t m, int64_t k, int64_t n, float alpha, float beta,
                          const fmm_options* opts);

/* Seeded input generator: out(i, j) = lo + (hi - lo) * u, u in [0, 1) from a
 * counter-based splitmix64 stream (element index i + j * rows), identical to
 * the host generator used by the tests. */
fmm_status fmm_fill_uniform(fmm_handle h, double* out, int64_t rows, int64_t cols, int64_t ld, uint64_t seed,
                            uint64_t stream, double lo, double hi);

/* max_ij |a_ij - b_ij| / |a_ij| (MaxRelativeDiff, linalg/linalg.hpp:280-295)
 * and max_ij |a_ij - b_ij|; blocks until the result is on the host. */
fmm_status fmm_max_relative_diff(fmm_handle h, const double* a, int64_t lda, const double* b, int64_t ldb,
                                 int64_t m, int64_t n, double* max_rel, double* max_abs);

/* Diagonal scaling types: the reference's unnamed enum OUTSIDE_INSIDE,
 * INSIDE_OUTSIDE, INSIDE, OUTSIDE (scaling/scaling.hpp:19-24). */
enum {
  FMM_SCALING_OUTSIDE_INSIDE = 0,
  FMM_SCALING_INSIDE_OUTSIDE = 1,
  FMM_SCALING_INSIDE = 2,
  FMM_SCALING_OUTSIDE = 3
};

/* Diagonal scaling of the operands before a product, replacing
 * Scaling<double>(A, B, num_steps, r_vals, s_vals, scaling_type)
 * (scaling/scaling.hpp:153-196).  A (m x k) and B (k x n), device
 * matrices, are scaled in place on the handle's stream; r (m) and s (n),
 * device arrays, are in/out: the outer maxima are multiplied into their
 * entries (UpdateVals, scaling.hpp:93-98).  Fill them with 1 for the
 * reference's fresh vectors (its resize(m, 1.0) keeps the entries of
 * vectors that arrive sized).
 * Each step is an outer scaling (rows of A by 1 / max|A(i,:)|, columns of B
 * by 1 / max|B(:,j)|) and/or an inner scaling (columns of A by 1 / z_l and
 * rows of B by z_l, z_l = sqrt(max|A(:,l)| / max|B(l,:)|)) in the order of
 * `type`.  Bit for bit the reference's result.  An unknown type returns
 * FMM_ERR_INVALID_ARGUMENT (the reference throws "Unknown iteration type."). */
fmm_status fmm_diagonal_scaling(fmm_handle h, double* A, int64_t lda, double* B, int64_t ldb, int64_t m, int64_t k,
                                int64_t n, int num_steps, int type, double* r, double* s);

/* C(i, j) := (C(i, j) * r[i]) * s[j] on the handle's stream, replacing
 * PostProcessScaling(C, r_vals, s_vals) (scaling/scaling.hpp:143-148): the
 * product of the scaled operands back to the product of the originals. */
fmm_status fmm_scaling_postprocess(fmm_handle h, double* C, int64_t ldc, int64_t m, int64_t n, const double* r,
                                   const double* s);

/* The two calls above with HOST matrices and factor vectors (copied in,
 * scaled on the device, copied back; they return when the results are on
 * the host): Scaling / PostProcessScaling over host buffers, for the C++
 * adapter (include/fmm/scaling.hpp). */
fmm_status fmm_diagonal_scaling_host(fmm_handle h, double* A, int64_t lda, double* B, int64_t ldb, int64_t m,
                                     int64_t k, int64_t n, int num_steps, int type, double* r, double* s);
fmm_status fmm_scaling_postprocess_host(fmm_handle h, double* C, int64_t ldc, int64_t m, int64_t n, const double* r,
                                        const double* s);

/* The four calls above with Scalar = float (Scaling<float>, as the
 * reference's scaling/fast_scaling.cpp uses it): maxima and products in
 * float, each 1.0 / max and sqrt(max / max) taken in double and rounded to
 * float as the reference's template does; bit for bit its result. */
fmm_status fmm_diagonal_scaling_f32(fmm_handle h, float* A, int64_t lda, float* B, int64_t ldb, int64_t m, int64_t k,
                                    int64_t n, int num_steps, int type, float* r, float* s);
fmm_status fmm_scaling_postprocess_f32(fmm_handle h, float* C, int64_t ldc, int64_t m, int64_t n, const float* r,
                                       const float* s);
fmm_status fmm_diagonal_scaling_f32_host(fmm_handle h, float* A, int64_t lda, float* B, int64_t ldb, int64_t m,
                                         int64_t k, int64_t n, int num_steps, int type, float* r, float* s);
fmm_status fmm_scaling_postprocess_f32_host(fmm_handle h, float* C, int64_t ldc, int64_t m, int64_t n,
                                            const float* r, const float* s);

/* Waits for all work queued on the handle's stream.  FMM_ERR_TIMEOUT if a
 * tensor-core kernel of a split-BF16 product gave up one of its bounded
 * waits since the last check (its results are then not valid). */
fmm_status fmm_synchronize(fmm_handle h);

/* Diagnostic of the bounded device waits (no counterpart in the reference):
 * launches one kernel whose mbarrier wait is never satisfied and must give
 * up after limit_ms; *code receives the error code it recorded (nonzero
 * when the timeout path works).  The handle's error word is cleared and the
 * context stays usable. */
fmm_status fmm_selftest_wait_timeout(fmm_handle h, double limit_ms, int* code);

/* Number of kernels the handle has launched since it was created. */
int64_t fmm_kernel_launch_count(fmm_handle h);

/* Per-phase timing (the reference times only the whole call,
 * algorithms/strassen.hpp:708-721).  While enabled, every launch of
 * fmm_fast_matmul / fmm_dgemm is bracketed by CUDA events on the handle's
 * stream; fmm_profile_read synchronises and returns the totals since the
 * last reset, with the algorithmic work of those launches: FLOPs of the
 * leaf and fringe products, and HBM bytes of the operand formations and
 * combinations counted as every input block read once and every output
 * block written once. */
typedef struct fmm_profile {
  int64_t form_launches, gemm_launches, peel_launches, combine_launches;
  double form_ms, gemm_ms, peel_ms, combine_ms;
  double form_bytes, combine_bytes;
  double gemm_flops, peel_flops;
  /* split leaf products (counted in gemm_* above as well): time of the
   * scale / split kernels within gemm_ms, and the tensor-core operations of
   * the slice products (2 m n k per product, S(S+1)/2 products per leaf;
   * BF16 FLOPs for SPLIT_BF16, INT8 operations for SPLIT_INT8) */
  double split_ms;
  double split_bf16_flops;
} fmm_profile;

fmm_status fmm_profile_enable(fmm_handle h, int enable);
fmm_status fmm_profile_reset(fmm_handle h);
fmm_status fmm_profile_read(fmm_handle h, fmm_profile* out);

/* ---- Batches, autotuning and CUDA-graph plans.  No counterpart in the
 * reference, which multiplies one pair per call and fixes the algorithm and
 * depth at compile time. */

/* Algorithm value of a batch item: -1 lets the autotuner choose the
 * algorithm and depth; FMM_ALG_CLASSICAL is one GEMM
 * C = alpha * A * B + beta * C (beta honoured). */
#define FMM_ALG_AUTO (-1)
#define FMM_ALG_CLASSICAL (-2)

typedef struct fmm_batch_item {
  int alg;        /* algorithm index, FMM_ALG_AUTO or FMM_ALG_CLASSICAL */
  int num_steps;  /* recursive levels (ignored for FMM_ALG_AUTO / FMM_ALG_CLASSICAL) */
  const double* A;
  int64_t lda;
  const double* B;
  int64_t ldb;
  double* C;
  int64_t ldc;
  int64_t m, k, n;
  double x, alpha, beta; /* as in fmm_fast_matmul */
  int precision;         /* fmm_precision of the item's leaf products (0 = FP64) */
  int split_slices;      /* slices: SPLIT_BF16 2..6, SPLIT_INT8 2..8 (0 = default) */
  int gemm_tile;         /* fmm_gemm_tile of the item's FP64 products (AUTO: the autotuned choice of
                            the item's shape bucket for FMM_ALG_AUTO items, else per problem) */
} fmm_batch_item;

/* Independent products in one program: the operand formations of all items
 * level by level (one launch per algorithm and level), the leaf products of
 * ALL items in one persistent grouped GEMM launch, then the combinations and
 * fringe products.  Each item's result equals the one fmm_fast_matmul gives
 * for it alone (bit for bit).  Items whose combined workspace exceeds the
 * handle's limit are run in several such programs.  Device pointers; queued
 * on the handle's stream. */
fmm_status fmm_fast_matmul_batched(fmm_handle h, const fmm_batch_item* items, int count);

/* The (algorithm, num_steps) the handle uses for FMM_ALG_AUTO items of this
 * shape: the autotuned choice of the shape's bucket (ceil(log2) of m, k and
 * n) if fmm_autotune measured it, otherwise a size rule (classical below
 * 4000; Strassen with 2 steps from 4000; fast424_26_206 with 2 steps from
 * 12000 in every dimension).  *alg is FMM_ALG_CLASSICAL for a plain GEMM. */
fmm_status fmm_autotune_choice(fmm_handle h, int64_t m, int64_t k, int64_t n, int* alg, int* num_steps);
/* The FP64 GEMM tile configuration (fmm_gemm_tile) the autotuner measured
 * fastest for the shape's bucket, FMM_GEMM_TILE_AUTO for an unmeasured
 * bucket.  FMM_ALG_AUTO batch items with gemm_tile AUTO use it. */
fmm_status fmm_autotune_tile(fmm_handle h, int64_t m, int64_t k, int64_t n, int* tile);

/* Times, for one representative shape per bucket of `shapes` (count x 3:
 * m, k, n), the classical GEMM and every candidate algorithm with 1 ..
 * max_steps levels (leaf blocks of at least 64), each with both FP64 GEMM
 * tile configurations, and records the fastest per bucket in the handle.  candidates may be NULL (Strassen, fast424_26_206,
 * fast333_23_125, smirnov333_23_128).  Allocates scratch matrices. */
fmm_status fmm_autotune(fmm_handle h, const int64_t* shapes, int count, const int* candidates, int n_candidates,
                        int max_steps);

/* The tuning table as text lines "mb kb nb alg steps tile" (buckets are
 * ceil(log2(dim)), tile an fmm_gemm_tile), and loading it back (lines
 * without the tile column load with FMM_GEMM_TILE_AUTO). */
fmm_status fmm_autotune_export(fmm_handle h, char* buf, size_t cap, size_t* len);
fmm_status fmm_autotune_import(fmm_handle h, const char* text);

/* A product or a batch planned once and captured as a CUDA graph; executing
 * replays the graph on the handle's stream (same pointers, current data).
 * The plan owns its workspace and descriptors. */
typedef struct fmm_plan_s* fmm_plan;
fmm_status fmm_plan_create(fmm_handle h, int alg, const double* A, int64_t lda, const double* B, int64_t ldb,
                           double* C, int64_t ldc, int64_t m, int64_t k, int64_t n, int num_steps, double x,
                           double alpha, double beta, const fmm_options* opts, fmm_plan* out);
fmm_status fmm_plan_create_batched(fmm_handle h, const fmm_batch_item* items, int count, fmm_plan* out);
fmm_status fmm_plan_execute(fmm_plan p);
fmm_status fmm_plan_destroy(fmm_plan p);
/* Kernels one execution launches. */
int64_t fmm_plan_kernel_count(fmm_plan p);

/* ---- Serving: a continuous-batching request loop (no counterpart in the
 * reference).  A background thread admits queued requests, in arrival
 * order, whenever a launch slot (one stream each) is free and the S/T/M
 * workspace of the request fits in the server's workspace pool; the
 * requests admitted together go out as one batch program on that slot's
 * stream, so work of different slots overlaps on the device.  Operands stay
 * where the caller put them (device memory); C is written in place.  Each
 * result equals the one fmm_fast_matmul (or the classical product) gives for
 * the request alone, bit for bit. */
typedef struct fmm_server_s* fmm_server;

typedef struct fmm_server_config {
  int device;
  size_t workspace_bytes; /* pool for in-flight S/T/M temporaries (0 = 40% of free memory) */
  int max_inflight;       /* launch slots / streams (0 = 4) */
  int max_batch;          /* requests per launch (0 = 64) */
} fmm_server_config;

typedef struct fmm_request {
  int alg;        /* algorithm index, FMM_ALG_AUTO or FMM_ALG_CLASSICAL */
  int num_steps;
  int precision;  /* fmm_precision */
  const double* A;
  int64_t lda;
  const double* B;
  int64_t ldb;
  double* C;
  int64_t ldc;
  int64_t m, k, n;
  double x, alpha, beta;
  int split_slices; /* slices: SPLIT_BF16 2..6, SPLIT_INT8 2..8 (0 = default) */
} fmm_request;

typedef struct fmm_request_info {
  int done;          /* 1 once C holds the result */
  fmm_status status; /* of the request's planning / launch */
  double submit_ms;  /* host clock (ms since the server started) at submission */
  double launch_ms;  /* ... when its batch was launched */
  double done_ms;    /* ... when its batch was seen complete */
} fmm_request_info;

typedef struct fmm_server_stats {
  int64_t submitted, completed, launches, batches;
  int64_t max_batch_seen;
  size_t workspace_peak;
} fmm_server_stats;

fmm_status fmm_server_create(const fmm_server_config* cfg, fmm_server* out);
fmm_status fmm_server_submit(fmm_server s, const fmm_request* req, uint64_t* ticket);
/* Waits up to timeout_ms (< 0: forever) for a request; FMM_ERR_TIMEOUT if it
 * is not done by then. */
fmm_status fmm_server_wait(fmm_server s, uint64_t ticket, double timeout_ms, fmm_request_info* info);
/* Waits up to timeout_ms (< 0: forever) until every submitted request is done. */
fmm_status fmm_server_drain(fmm_server s, double timeout_ms);
fmm_status fmm_server_get_stats(fmm_server s, fmm_server_stats* out);
/* Stops the loop after the in-flight work finishes; pending requests are
 * dropped with FMM_ERR_TIMEOUT. */
fmm_status fmm_server_destroy(fmm_server s);

/* Allocation-free FastMatmul.  No counterpart in the reference.
 *
 * For callers that may not allocate device memory at all: code whose device
 * memory belongs to another framework's pool or to a fixed budget, and
 * latency-critical loops where cudaMalloc's implicit device synchronisation
 * is not acceptable.  The call computes exactly what fmm_fast_matmul
 * computes, with the same kernels, but takes its workspace and launch
 * descriptors from a static device array of FMM_NOALLOC_SCRATCH_BYTES that
 * the library defines; it needs no handle and calls no cudaMalloc,
 * cudaFree, pinned-host allocation or other device-allocating routine
 * (host-side planning uses ordinary heap memory).
 *
 *  - Limit: every GPU that loads the library holds the 64 MiB array until
 *    the process exits; 1 MiB of it holds launch descriptors, the rest the
 *    S/T/M temporaries.  The call picks the most breadth-first schedule that
 *    fits and returns FMM_ERR_WORKSPACE_TOO_SMALL, with the sizes in
 *    fmm_last_error(), when even the depth-first one does not (for
 *    Strassen with one step: dimensions up to about 1400).
 *  - The first call on a device looks up the array's device address (with
 *    that device current); make that first call before any stream capture.
 *  - The launch descriptors are copied from a host buffer that the next call
 *    reuses, so a stream in capture mode is refused with
 *    FMM_ERR_NOT_SUPPORTED before anything is queued on it.
 *  - Every call shares the array and it keeps the last call's contents;
 *    nothing in it has to start at zero.  Calls that overlap on the GPU
 *    (different streams, or several host threads) race on it.
 *  - Device pointers on the current device; the work is queued on `stream`
 *    (a cudaStream_t, NULL = legacy default) and the call returns once it is
 *    queued (copying the launch descriptors from host memory may first wait
 *    for earlier work on that stream). */
#define FMM_NOALLOC_SCRATCH_BYTES ((size_t)64 << 20)
fmm_status fmm_fast_matmul_noalloc(int alg, const double* A, int64_t lda, const double* B, int64_t ldb, double* C,
                                   int64_t ldc, int64_t m, int64_t k, int64_t n, int num_steps, double x,
                                   double alpha, double beta, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FMM_H_ */
