/*
 * laker_b200.h - C ABI of liblaker_b200.so, the B200 (sm_100a) implementation
 * of the LAKER exact-kernel solve path:
 *
 *   - the matrix-free attention-kernel operator  A = lambda*I + exp(E E^T)
 *     applied to PositionEmbedding outputs E (n x d, d <= 16),
 *   - the preconditioned conjugate gradient loop (single and batched RHS),
 *   - application of the factored CCCP preconditioner
 *     P = c^-1/2 I + Q V diag(lambda_i^-1/2 - c^-1/2) V^T Q^T.
 *
 * Conventions
 *   - Every pointer argument is DEVICE memory unless stated otherwise.  The
 *     caller owns (allocates and frees) every buffer, including workspaces;
 *     the library never calls cudaMalloc/cudaFree.  Workspace sizes come from
 *     the matching *_workspace_bytes query.
 *   - Matrices are row-major with an explicit leading dimension (elements).
 *   - `stream` is a cudaStream_t (NULL = legacy default stream).  Calls are
 *     asynchronous on that stream except laker_pcg_solve, which synchronises
 *     the stream to poll convergence and returns when the solve has ended.
 *   - Every entry point returns a laker status code (0 = LAKER_OK).  Kernels
 *     never trap.  A device-side failure (a bounded wait that expired) is
 *     recorded in the status word at the start of the call's workspace (or of
 *     the allocation-free entry point's scratch): the asynchronous products
 *     then write NaN to every output element, laker_workspace_status /
 *     laker_noalloc_status read the word back after the stream synchronises,
 *     and the synchronising calls (laker_pcg_solve, the engine) return it as
 *     their status.
 *
 * Reference interfaces cited as path:line are in the LAKER Python package
 * (laker/kernels.py, laker/solvers.py, laker/preconditioner.py, laker/core.py).
 */
#ifndef LAKER_B200_H
#define LAKER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status codes                                                              */
/* ------------------------------------------------------------------------ */
enum laker_status {
  LAKER_OK = 0,
  LAKER_ERR_INVALID_ARG = 1,   /* bad size, NULL pointer, misaligned buffer  */
  LAKER_ERR_CUDA = 2,          /* a CUDA runtime call failed                 */
  LAKER_ERR_BREAKDOWN = 3,     /* PCG: p^T A p <= -eps ||p|| ||Ap||          */
  LAKER_ERR_NOT_CONVERGED = 4, /* PCG: max_iter reached (x is still valid)   */
  LAKER_ERR_NONFINITE = 5,     /* PCG: NaN/Inf in an inner product           */
  LAKER_ERR_TIMEOUT = 6,       /* a bounded device wait expired              */
  LAKER_ERR_WORKSPACE = 7,     /* workspace smaller than the query returned  */
  LAKER_ERR_UNSUPPORTED = 8,   /* shape/dtype combination not implemented    */
  LAKER_ERR_SCRATCH_LIMIT = 9, /* larger than the fixed scratch of the
                                  allocation-free entry point               */
  LAKER_ERR_CAPACITY = 10      /* engine: no free slot, points or pairs      */
};

/* Library version as 10000*major + 100*minor + patch. */
int laker_version(void);

/* Human-readable name of a status code (static storage). */
const char* laker_status_string(int status);

/* cudaError_t of the most recent LAKER_ERR_CUDA on the calling thread. */
int laker_last_cuda_error(void);

/* Device status word of the last call that used `workspace` (a workspace of
 * laker_attn_matvec_f32 / _f64): synchronises `stream` and writes LAKER_OK or
 * the device-side failure (LAKER_ERR_TIMEOUT) to *status.  The outputs of a
 * failed call are NaN.  No counterpart in the reference, whose products are
 * synchronous torch calls that raise (laker/solvers.py:343-352 raises on
 * breakdown). */
int laker_workspace_status(const void* workspace, int* status, void* stream);

/* ------------------------------------------------------------------------ */
/* Embedding layouts                                                         */
/* ------------------------------------------------------------------------ */
/* The kernels read embeddings in two packed layouts produced on the device:
 *   packed32: FP32, point pairs interleaved per dimension
 *             block q = {e[2q][0], e[2q+1][0], e[2q][1], e[2q+1][1], ...},
 *             dimension padded to an even count, pair count padded to whole
 *             256-column tiles with zero points;
 *   packed64: FP64, one row per point (dimension padded to even), row count
 *             padded to whole 128-row tiles with zero points.
 * `E` is an (n x d) row-major matrix with leading dimension ld >= d, either
 * float (e_is_f64 = 0) or double (e_is_f64 = 1).  1 <= d <= 16.
 */
size_t laker_packed32_floats(int64_t n, int d);
size_t laker_packed64_doubles(int64_t n, int d);
int laker_pack_f32(const void* E, int e_is_f64, int64_t n, int d, int64_t ld, float* packed32,
                   void* stream);
int laker_pack_f64(const void* E, int e_is_f64, int64_t n, int d, int64_t ld, double* packed64,
                   void* stream);

/* ------------------------------------------------------------------------ */
/* Attention-kernel operator                                                 */
/* ------------------------------------------------------------------------ */
/* Workspace for laker_attn_matvec_f32 / _f64 (partial row sums of the column
 * segments).  precision is 32 or 64. */
size_t laker_matvec_workspace_bytes(int64_t m, int64_t n, int d, int k, int precision);

/* FP32 fused matvec ("sloppy" operator used inside the PCG loop).
 *   Y = lam * X[:m] + exp(Er Ec^T) X          (X: n x k, Y: m x k)
 * Er/Ec are packed32 buffers of m and n points.  lam is applied only when
 * m == n (pass 0 for a rectangular product such as prediction).  clamp = 1
 * clamps the Gram entry at 80 before exp, as the reference does when
 * max ||e||^2 >= 80.  The n x n kernel matrix is never stored.
 * Replaces AttentionKernelOperator.matvec / matvec_impl
 * (laker/kernels.py:187-270) and dense_attention_matvec (kernels.py:121-130)
 * for float32 operators. */
int laker_attn_matvec_f32(const float* rows32, int64_t m, const float* cols32, int64_t n, int d,
                          float lam, int clamp, const float* X, int k, int64_t ldx, float* Y,
                          int64_t ldy, void* workspace, size_t workspace_bytes, void* stream);

/* Algorithmic work of one square FP32 operator application (the kernel
 * laker_attn_matvec_f32 and laker_pcg_solve use for n points of dimension d):
 * kernel entries evaluated, FP32 flops (2 per FMA: d logit FMAs plus one
 * accumulation FMA per use of an entry) and exp2 evaluations.  With the
 * symmetric kernel each off-diagonal entry is evaluated once and used twice.
 * No counterpart in the reference (roofline accounting). */
int laker_fp32_matvec_work(int64_t n, int d, double* entries, double* flops, double* exps);

/* Which kernel a square FP32 operator application of n points of dimension
 * d runs: 0 the plain fused kernel (always for n of at most
 * LAKER_VARIANT_SYM_MIN_BLOCKS x 512 points, default 3072, where the
 * symmetric kernels have too few block pairs to fill the GPU), 1 the
 * symmetric kernel with logits on the CUDA cores, 2 the symmetric kernel with
 * logits on the tensor cores (split-FP16 or split-TF32 tcgen05 MMAs,
 * LAKER_VARIANT_K1T_LOGITS; then `flops` above counts only the CUDA-core
 * accumulation FMAs and the logits add 3 x 2 x 16 tensor flops per entry
 * evaluated); -1 for invalid arguments.  No counterpart in the reference. */
int laker_fp32_operator_kernel(int64_t n, int d);

/* Kernel variant choices, changeable between calls (no call may be in flight
 * on any stream): they start from the environment switches and are what the
 * autotuner sets after timing the candidates on the caller's problem size.
 *   LAKER_VARIANT_K1T_UNIT       TMEM unit of the tensor-core symmetric
 *                                operator: 4 (default) or 2 row tiles
 *   LAKER_VARIANT_K2_LOGITS_N32  multi-RHS chunks of <= 32 right-hand sides,
 *   LAKER_VARIANT_K2_LOGITS_N128 of 33..128, and
 *   LAKER_VARIANT_K2_LOGITS_WIDE of more than 128: 0 logits on the CUDA cores
 *                                (default), 1 logits on the tensor cores
 *   LAKER_VARIANT_K1T_LOGITS     operands of the tensor-core symmetric
 *                                operator's logits: 0 split TF32, 1 split
 *                                FP16 (default; three kind::f16 products of
 *                                K = 16; unclamped operators only, clamped
 *                                ones keep split TF32).  An engine keeps the
 *                                format it was initialised with.
 *   LAKER_VARIANT_SYM_MIN_BLOCKS square FP32 operators (single solves and
 *                                matvecs; not the batched engine) of at most
 *                                this many 512-point blocks take the plain
 *                                kernel: 0..64, default 6
 * laker_set_variant returns the previous value, or -1 (nothing changed) for
 * an unknown `which` or an invalid value; laker_get_variant returns the
 * current value (-1 for an unknown `which`).  No counterpart in the
 * reference. */
#define LAKER_VARIANT_K1T_UNIT 0
#define LAKER_VARIANT_K2_LOGITS_N32 1
#define LAKER_VARIANT_K2_LOGITS_N128 2
#define LAKER_VARIANT_K2_LOGITS_WIDE 3
#define LAKER_VARIANT_SYM_MIN_BLOCKS 4
#define LAKER_VARIANT_K1T_LOGITS 5
/*   LAKER_VARIANT_WAIT_LIMIT_US  time limit of the kernels' bounded pipeline
 *                                waits in microseconds, 0..2000000 (default
 *                                2000000).  It applies on the current device
 *                                (set it once per device).  0 makes every
 *                                pipeline wait give up at once: the kernels
 *                                then drain their copies and tensor-core
 *                                operations in flight (always with the full
 *                                limit), record LAKER_ERR_TIMEOUT and return,
 *                                which runs the failure path deterministically
 *                                without a fault or a hang. */
#define LAKER_VARIANT_WAIT_LIMIT_US 6
/*   LAKER_VARIANT_MULTI_FLASH_K  multi-RHS FP32 products of unclamped
 *                                operators with at most this many right-hand
 *                                sides take the flash-style tensor-core kernel
 *                                (logits and P X on the tensor cores, P kept
 *                                in tensor memory; chunks of 32 right-hand
 *                                sides); 0 turns it off.  Default 32
 *                                (environment LAKER_MULTI_FLASH_K). */
#define LAKER_VARIANT_MULTI_FLASH_K 7
int laker_set_variant(int which, int value);
int laker_get_variant(int which);

/* Allocation-free FP32 fused matvec (single right-hand side).
 *   y = lam * x[:m] + exp(Er Ec^T) x          (x: n, y: m)
 * Same arguments and result as laker_attn_matvec_f32 with k = 1, but without
 * a workspace: it is for callers that hold device buffers yet cannot allocate
 * device memory (a host that only receives buffers from another framework's
 * allocator, or a loop where cudaMalloc's implicit synchronisation and pool
 * growth are not allowed).  Its scratch is a fixed array of
 * LAKER_NOALLOC_SCRATCH_BYTES inside the library, held by every GPU that loads
 * it until the process exits; m must not exceed LAKER_NOALLOC_MAX_ROWS
 * (LAKER_ERR_SCRATCH_LIMIT otherwise).  The first call on each device sets the
 * array up (symbol lookup, possibly loading the module): make it before any
 * stream capture.  Every call reuses the same array, so calls that overlap on
 * the GPU (other streams, unordered host threads) race.  It calls no
 * allocation routine.  This entry point has no counterpart in the reference. */
#define LAKER_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)
#define LAKER_NOALLOC_MAX_ROWS 2000000
int laker_attn_matvec_f32_noalloc(const float* rows32, int64_t m, const float* cols32, int64_t n,
                                  int d, float lam, int clamp, const float* x, float* y,
                                  void* stream);

/* Device status word of the last laker_attn_matvec_f32_noalloc call on the
 * current device (the word lives in the fixed scratch array): synchronises
 * `stream` and writes LAKER_OK or LAKER_ERR_TIMEOUT to *status; a failed call
 * wrote NaN to y.  It allocates nothing.  Like the entry point it reports on,
 * it has no counterpart in the reference. */
int laker_noalloc_status(int* status, void* stream);

/* FP64 fused matvec / residual ("accurate" operator: FP64 logits, FP64 exp,
 * FP64 accumulation).
 *   Y = B - (lam * X[:m] + exp(Er Ec^T) X)    if B != NULL
 *   Y =      lam * X[:m] + exp(Er Ec^T) X     otherwise
 * Er/Ec are packed64 buffers.  Used for the true-residual recomputation of
 * the PCG loop and for float64 operators and predictions.
 * Replaces the float64 path of AttentionKernelOperator.matvec
 * (laker/kernels.py:187-270), the residual replacement r = b - A x
 * (laker/solvers.py:264) and the exact-kernel prediction loop
 * (laker/core.py:633-655). */
int laker_attn_matvec_f64(const double* rows64, int64_t m, const double* cols64, int64_t n, int d,
                          double lam, int clamp, const double* X, int k, int64_t ldx,
                          const double* B, int64_t ldb, double* Y, int64_t ldy, void* workspace,
                          size_t workspace_bytes, void* stream);

/* diag(A) = lam + exp(||e_i||^2) in FP64.
 * Replaces AttentionKernelOperator.diagonal (laker/kernels.py:272-283). */
int laker_attn_diagonal(const double* packed64, int64_t n, int d, double lam, double* out,
                        void* stream);

/* Materialised kernel block K = exp(Er Ec^T) (m x p), FP32 or FP64 output
 * (out_is_f64), computed from the packed64 embeddings with FP64 logits.
 * Replaces AttentionKernelOperator.kernel_eval (laker/kernels.py:301-354). */
int laker_kernel_eval(const double* rows64, int64_t m, const double* cols64, int64_t p, int d,
                      int clamp, void* out, int out_is_f64, int64_t ldo, void* stream);

/* ------------------------------------------------------------------------ */
/* Factored CCCP preconditioner                                              */
/* ------------------------------------------------------------------------ */
typedef struct laker_precond {
  const float* q_basis; /* (n x ldq) row-major, orthonormal columns Q in the
                           first nr columns, zeros after; 16-byte aligned     */
  const float* w_core;  /* (nr x nr) row-major W = V diag(l^-1/2 - c^-1/2) V^T */
  int64_t n;
  int nr;               /* 1 <= nr <= 1024                                   */
  int ldq;              /* leading dimension of q_basis: multiple of 4, >= nr */
  double inv_sqrt_iso;  /* c^-1/2, c = isotropic coefficient                 */
} laker_precond;

size_t laker_precond_workspace_bytes(int64_t n, int nr, int k);

/* Z = P R = c^-1/2 R + Q W Q^T R for R (n x k), FP64 in, FP32 or FP64 out
 * (k > 1: ldr = ldz = k).
 * Replaces preconditioner_apply_core / CCCPPreconditioner.apply
 * (laker/preconditioner.py:52-68, :286-310). */
int laker_precond_apply(const laker_precond* pc, const double* R, int k, int64_t ldr, void* Z,
                        int z_is_f64, int64_t ldz, void* workspace, size_t workspace_bytes,
                        void* stream);

/* ------------------------------------------------------------------------ */
/* Preconditioned conjugate gradient                                         */
/* ------------------------------------------------------------------------ */
typedef struct laker_operator {
  const float* packed32;  /* packed32 embeddings (sloppy FP32 operator)     */
  const double* packed64; /* packed64 embeddings (accurate FP64 operator)   */
  int64_t n;
  int d;
  double lambda_reg;
  int clamp;
} laker_operator;

typedef struct laker_pcg_params {
  double tol;            /* stop when ||b - A x||_F <= tol ||b||_F (FP64 A)  */
  int max_iter;          /* iteration cap (reference default: n)           */
  double reliable_delta; /* FP64 residual recomputed when the recurrence
                            residual fell by this factor since the last
                            recomputation (the Python solver passes 0.03)  */
  double breakdown_eps;  /* breakdown test p^T A p <= -eps ||p|| ||Ap||     */
  int check_every;       /* host polls the device status every N iterations */
  int has_x0;            /* 1: X holds the initial guess on entry           */
  int profile;           /* 1: time the fused matvec launches with events   */
  int column_stop;       /* k > 1 only.  0: stop when ||B - A X||_F <= tol
                            ||B||_F (the reference's global test); 1: each
                            column stops on its own FP64 residual
                            ||b_c - A x_c|| <= tol ||b_c|| and is frozen,
                            the solve ends when every column has          */
} laker_pcg_params;

typedef struct laker_pcg_result {
  int status;              /* LAKER_OK / _BREAKDOWN / _NOT_CONVERGED / ...  */
  int iterations;          /* PCG iterations (FP32 operator applications)   */
  int accurate_matvecs;    /* FP64 residual recomputations                  */
  double residual_norm;    /* ||b - A x||_F of the returned x (FP64 A)      */
  double rhs_norm;         /* ||b||_F                                       */
  double recurrence_norm;  /* last recurrence residual norm                 */
  int kernel_launches;     /* kernels this call launched (all of them)      */
  double fp32_matvec_ms;   /* profile: summed device time of FP32 matvecs   */
  double fp64_matvec_ms;   /* profile: summed device time of FP64 matvecs   */
  int fp32_matvec_launches;
  int fp64_matvec_launches;
} laker_pcg_result;

size_t laker_pcg_workspace_bytes(int64_t n, int d, int nr, int k);

/* Solves A X = B for k right-hand sides (B, X: n x k row-major, ld = k) with
 * mixed-precision PCG: FP32 fused operator inside the iteration (k = 1: the
 * symmetric single-RHS kernels; k > 1: the multi-RHS operator), FP64
 * vectors, inner products and scalars on the device, and reliable updates
 * that replace the recurrence residual by the FP64 residual B - A X; the stop
 * test is on that FP64 residual.  For k > 1 alpha and beta are per column,
 * a breakdown in any column ends the solve, and the stop test is the
 * Frobenius one of solve_2d unless params->column_stop asks for per-column
 * stops.  `pc` may be NULL (identity preconditioner).  Every decision of an
 * iteration is taken on the device; the call captures one iteration as a
 * CUDA graph on a private stream, replays it on `stream`, polls the device
 * state every check_every iterations (0: about every 10 ms of work) and
 * returns when the solve has ended (so it cannot itself be captured into a
 * caller's graph).  With `profile` (k = 1) the kernels are launched one by
 * one and the operator launches timed.  A device-side failure of a kernel
 * (LAKER_ERR_TIMEOUT) ends the solve and is returned.  Replaces
 * PreconditionedConjugateGradient.solve / solve_1d / solve_2d
 * (laker/solvers.py:130-394). */
int laker_pcg_solve(const laker_operator* op, const laker_precond* pc, const double* B, int k,
                    double* X, const laker_pcg_params* params, void* workspace,
                    size_t workspace_bytes, laker_pcg_result* result, void* stream);

/* ------------------------------------------------------------------------ */
/* Solve engine: many independent regressions in one device loop            */
/* ------------------------------------------------------------------------ */
/* A persistent device loop over resident instances ("slots").  Per
 * iteration: one symmetric FP32 matvec launch over the block pairs of the
 * running instances (the list is compacted on the device after every
 * iteration, so the whole grid works on what is left), vector kernels over
 * the 512-point blocks of every running instance with per-instance reductions
 * in a fixed order, and a symmetric FP64 residual over the instances whose
 * recurrence asked for one; scalars and convergence masks live on the device
 * and the iteration is captured once as a CUDA graph.  Instances are admitted
 * and collected between graph replays (continuous batching); an instance's
 * result does not depend on the other instances in the engine.  The caller
 * owns both the host state buffer and the device workspace; the engine
 * allocates nothing.  One host thread drives an engine.
 * Replaces loops of PreconditionedConjugateGradient.solve calls
 * (laker/solvers.py:130-295) over independent problems; the reference has no
 * engine of its own. */
typedef struct laker_engine_config {
  int max_slots;       /* instances resident at once                            */
  int64_t max_points;  /* sum over resident instances of round_up(n, 512)       */
  int64_t max_pairs;   /* sum over resident instances of nb (nb + 1) / 2,
                          nb = ceil(n / 512)                                    */
  int d;               /* embedding dimension (all instances)                   */
  int max_nr;          /* largest preconditioner N_r (0: none)                  */
  int clamp;           /* 1: clamp Gram entries (needed when any instance's
                          operator does not skip the clamp)                     */
  int chunk;           /* iterations per graph replay (>= 1)                    */
} laker_engine_config;

size_t laker_engine_host_bytes(const laker_engine_config* cfg);
size_t laker_engine_workspace_bytes(const laker_engine_config* cfg);

/* Sets up an engine in `host` (host memory, laker_engine_host_bytes) over
 * `workspace` (device memory, laker_engine_workspace_bytes).  params: tol,
 * max_iter, reliable_delta, breakdown_eps as for laker_pcg_solve (has_x0
 * must be 0).  All later calls enqueue on `stream`. */
int laker_engine_init(void* host, size_t host_bytes, void* workspace, size_t workspace_bytes,
                      const laker_engine_config* cfg, const laker_pcg_params* params,
                      void* stream);

/* Admits one instance: n points, lambda, its packed32 / packed64 embeddings
 * (laker_pack_f32 / _f64 layouts, DEVICE), preconditioner (HOST struct of
 * device factors, or NULL) and right-hand side b (DEVICE, n doubles).  The
 * embeddings and b are copied into the engine; the factors must stay alive
 * until the instance is collected.  Writes the slot index to *slot.
 * LAKER_ERR_CAPACITY when no slot, points or pairs are free (after
 * compacting the resident instances). */
int laker_engine_admit(void* host, int64_t n, double lambda_reg, const float* packed32,
                       const double* packed64, const laker_precond* pc, const double* b,
                       int* slot);

/* Runs one graph replay (cfg.chunk iterations of every running instance) and
 * waits for it.  *running: instances still iterating afterwards. */
int laker_engine_step(void* host, int* running);

/* laker_engine_step in two halves: _launch enqueues the replay and the read
 * back of the engine's flags into the host state, _sync waits for them and
 * updates the stopped slots; admit and collect are refused in between.
 * _launch returns at once only when the host state buffer is pinned
 * (cudaHostAlloc / cudaHostRegister); with pageable memory the read back
 * makes it wait for the replay. */
int laker_engine_launch(void* host);
int laker_engine_sync(void* host, int* running);

/* Slots that have stopped (converged, failed or hit max_iter) and are not yet
 * collected: up to max_slots of them into slots[], their number in *count. */
int laker_engine_finished(void* host, int* slots, int max_slots, int* count);

/* Copies the solution of a stopped slot to x (DEVICE, n doubles), fills
 * *result and frees the slot. */
int laker_engine_collect(void* host, int slot, double* x, laker_pcg_result* result);

/* Releases the engine's CUDA graph and private stream (the host and device
 * buffers stay the caller's). */
int laker_engine_release(void* host);

/* ---- one-shot batch on top of the engine ------------------------------- */
/* Instance k has n[k] points; every batched vector and packed buffer holds
 * instance k at points [offsets[k], offsets[k] + n[k]) with offsets[0] = 0 and
 * offsets[k+1] = offsets[k] + round_up(n[k], 256) (zero padding between).
 * laker_batch_layout fills offsets[0..count] (host array) and returns the
 * total padded length. */
int64_t laker_batch_layout(int count, const int64_t* n, int64_t* offsets);

typedef struct laker_batch {
  int count;                    /* instances                                   */
  int d;                        /* embedding dimension (all instances)         */
  int clamp;                    /* 1: clamp Gram entries (see attn_matvec)     */
  const int64_t* n;             /* HOST [count]: points per instance (>= 1)    */
  const double* lambda_reg;     /* HOST [count]                                */
  const float* packed32;        /* DEVICE: packed32 of instance k at float
                                   offset offsets[k] * round_up(d, 2)          */
  const double* packed64;       /* DEVICE: packed64 of instance k at double
                                   offset offsets[k] * round_up(d, 2)          */
  const laker_precond* precond; /* HOST [count] (device factors) or NULL       */
} laker_batch;

/* Workspace for a batch whose preconditioners have at most max_nr probes
 * (0: no preconditioner); 0 for invalid sizes.  Includes the engine's
 * workspace and a host-state area at its end. */
size_t laker_pcg_batched_workspace_bytes(int count, const int64_t* n, int d, int max_nr);

/* Solves A_k x_k = b_k for every instance: one engine sized for the batch,
 * every instance admitted, steps until all have stopped, every instance
 * collected.  B, X: batched vectors (padded length).  results: HOST array of
 * count results.  Returns LAKER_OK unless a call failed; per-instance
 * outcomes are in results[k].status.  Warm starts (has_x0) are not
 * supported. */
int laker_pcg_solve_batched(const laker_batch* batch, const double* B, double* X,
                            const laker_pcg_params* params, void* workspace,
                            size_t workspace_bytes, laker_pcg_result* results, void* stream);

/* ------------------------------------------------------------------------ */
/* Predictive variance                                                       */
/* ------------------------------------------------------------------------ */
/* var_q = max(0, exp(||e_q||^2) - sum_i Kxq[i, q] * V[i, q]) for q < m, with
 * Kxq, V (n x m) row-major FP64 and Eq the packed64 query embeddings.
 * Replaces laker/core.py:754-758 and :777 without the m x m kernel_eval. */
int laker_variance_finalize(const double* q64, int64_t m, int d, const double* Kxq,
                            const double* V, int64_t n, int64_t ld, double* var, void* stream);

/* ------------------------------------------------------------------------ */
/* Roofline denominators                                                     */
/* ------------------------------------------------------------------------ */
/* Measures, on the current device, the sustained FP32 FMA rate (TFLOP/s,
 * 2 flops per FMA), the MUFU exp2 rate (Tops/s) and the FP64 FMA rate
 * (TFLOP/s) with short register-resident microkernels (~50 ms).  `scratch`
 * must hold laker_peaks_scratch_bytes() bytes. */
size_t laker_peaks_scratch_bytes(void);
int laker_measure_peaks(void* scratch, double* ffma_tflops, double* mufu_tops,
                        double* dfma_tflops, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LAKER_B200_H */
