/*
 * jkogb.h -- C ABI of libjkogb_b200.so: the J-Kogbetliantz hyperbolic SVD step loop
 * of venovako/JKogb (real djk and complex zjk) on an NVIDIA B200 (sm_100a).
 *
 * The entry points replace the Fortran seam the reference's drivers call:
 *   DSTEP_LOOP(N, U, LDU, A, LDA, Z, LDZ, J, SIGMA, NN, P, Q, R, NM, DZ, N_2, STEP, TT, W, INFO)
 *     src/D/dstep.F90:472-604, called from src/D/djk.F90:83
 *   ZSTEP_LOOP(...)  src/Z/zstep.F90:482-615, called from src/Z/zjk.F90
 * together with the strategy plug-ins DPROC_INIT selects (src/D/dstep.F90:76-134):
 * ID_NCP 0/1/2 (greedy non-colliding selection, AW_NCP1 == AW_NCP2), 3 (AW_NCP3, the best
 * of the greedy walks from every start offset, src/shared/atypes.F90:488-592; its work
 * grows as N^4 per step, so N <= 256) and ID_TRU 0/1/2 (pair enumeration; the
 * selection is a total order, so it does not change results).
 * The caller's workspaces of the Fortran interface (NN, P, Q, NM, DZ, STEP, TT, W) live
 * on the device and are not arguments here.
 *
 * Conventions: column-major matrices with a leading dimension; complex matrices are
 * interleaved (re, im) doubles, the memory layout of Fortran COMPLEX(KIND=8); J holds
 * the N signs (+1/-1) as int.  Return value INFO as DSTEP_LOOP's: >= 0 the number of
 * steps with transformations, < 0 an error (see jk_strerror).  On return A holds the
 * final matrix with a zeroed diagonal, SIGMA its diagonal (the hyperbolic singular
 * values), U the accumulated left rotations and Z the inverse of the accumulated right
 * transformation, J Z^T J (real) / J Z^H J (complex), so that Y = U diag(SIGMA) Z.
 */
#ifndef JKOGB_H
#define JKOGB_H

#ifdef __cplusplus
extern "C" {
#endif

/* Options; a NULL pointer means all defaults (zero). */
typedef struct {
  int max_steps;    /* stop after this many steps (0: no limit, as DSTEP_LOOP, src/D/dstep.F90:564-578,
                       except in the batched solver, see JK_BATCH_STEP_BOUND); INFO = JK_ERR_MAX_STEPS
                       when hit, with A, U, Z, SIGMA as the loop left them */
  int zba_quirk;    /* complex BA branch of src/Z/ztransf.F90:325: 0 = as the reference (R1), 1 = R2 as the real code */
  int graph_steps;  /* steps per CUDA-graph launch (0: 32; -1: plain stream launches) */
  int device;       /* CUDA device ordinal for the host-pointer entry points (-1 or 0: current) */
  int reserved[4];
} jk_opts;

/* Optional per-step trace, the stderr CSV of DSTEP_EXEC (src/D/dstep.F90:389-442) and
 * the selected pivots of every step (the AW_OUT dump, src/shared/atypes.F90:30-77).
 * Host buffers sized by the caller; unused pointers may be NULL. */
typedef struct {
  int max_steps;        /* capacity of sl/nl/trig/hyp/tw/rounds */
  int *sl, *nl, *trig, *hyp;
  double *tw;
  int *rounds;          /* matching rounds of the selection of each step (telemetry) */
  long long max_piv;    /* capacity of piv in pivots */
  int *piv;             /* 2 ints per pivot: p, q (1-based), in selection order, all steps */
  long long n_piv;      /* out */
  int n_steps;          /* out: steps recorded (including the last, empty one) */
} jk_trace;

#define JK_ERR_CUDA (-30)       /* a CUDA runtime error */
#define JK_ERR_NOMEM (-31)      /* device allocation failed */
#define JK_ERR_TOO_LARGE (-32)  /* N beyond this build's limit (see jk_max_order; 256 for ID_NCP = 3) */
#define JK_ERR_ID_NCP (-21)     /* ID_NCP outside 0..3 */
#define JK_ERR_ID_TRU (-22)     /* ID_TRU outside 0..2 */
#define JK_ERR_J (-23)          /* a J entry is not +1 or -1 (TRU1/TRU2, src/shared/jstep.F90:38-39) */
#define JK_ERR_MAX_STEPS (-24)  /* opts->max_steps reached */
#define JK_ERR_NO_DEVICE (-33)  /* no CUDA device */
#define JK_ERR_SCRATCH (-34)    /* N beyond JK_NOALLOC_MAX_N (jk_dweights_noalloc) */
#define JK_ERR_STALL (-26)      /* internal: the device loop neither advanced nor ended (a library fault) */
#define JK_ERR_STATE (-27)      /* a jk_solver call out of order (advance or finish before begin) */

/* DSTEP_LOOP with host buffers, src/D/dstep.F90:472-604 (copies to and from the device).
 * A is in/out; U, Z, SIGMA are out.  N_2 is clamped as JSTEP_LEN does (src/shared/jstep.F90:124). */
int jk_dstep_loop(int n, double *U, int ldu, double *A, int lda, double *Z, int ldz, const int *J,
                  double *sigma, int n_2, int id_ncp, int id_tru, const jk_opts *opts, jk_trace *trace);

/* ZSTEP_LOOP with host buffers, src/Z/zstep.F90:482-615; U, A, Z are complex (2 doubles each). */
int jk_zstep_loop(int n, double *U, int ldu, double *A, int lda, double *Z, int ldz, const int *J,
                  double *sigma, int n_2, int id_ncp, int id_tru, const jk_opts *opts, jk_trace *trace);

/* The same loops on device buffers (leading dimension n), enqueued on `stream`
 * (a cudaStream_t, NULL = the default stream); J is a host array.  Synchronises the
 * stream before returning INFO.  Device buffers must be aligned as cudaMalloc returns them:
 * 8 bytes for real data, 16 for complex data and for A of a scored real solve
 * (jk_dstep_loop_dev_scored).  A NULL or misaligned U, A, Z or SIGMA returns -2, -4, -6
 * or -9, its position in DSTEP_LOOP's argument list, before anything runs on the device;
 * the same check makes jk_solver_begin / resume / finish return -2, jk_handle_weights and
 * the jk_batch_run / jk_batch_tune buffers -1. */
int jk_dstep_loop_dev(int n, double *dU, double *dA, double *dZ, const int *J, double *dsigma,
                      int n_2, int id_ncp, int id_tru, const jk_opts *opts, jk_trace *trace, void *stream);
int jk_zstep_loop_dev(int n, double *dU, double *dA, double *dZ, const int *J, double *dsigma,
                      int n_2, int id_ncp, int id_tru, const jk_opts *opts, jk_trace *trace, void *stream);

/* The same loop as a reusable object that can be advanced a given number of steps at a
 * time: the caller-owned workspace of DSTEP_LOOP (DZ, STEP, W, P, Q: src/D/djk.F90:47-56)
 * made once per order N, sign vector J, N_2 and strategy, and the loop of
 * src/D/dstep.F90:564-583 split at step boundaries.  Results are those of
 * jk_dstep_loop_dev / jk_zstep_loop_dev, whatever the split.
 *   create   the device workspace (J a host array; opts: max_steps, zba_quirk,
 *            graph_steps, device); NULL on error with *info set
 *   begin    a new solve on device buffers (leading dimension n, complex: interleaved):
 *            A in/out, U and Z out; enqueues U = Z = I and the loop-state reset on `stream`
 *   resume   a solve that an earlier loop left unfinished after `steps` steps (INFO
 *            JK_ERR_MAX_STEPS): A, U, Z as that loop returned them (diagonal in SIGMA,
 *            Z already J Z^T J); restores the loop's state from them and continues, so
 *            that the final results equal one uninterrupted solve's
 *   advance  runs the loop until S has grown by `steps` (0: until the loop ends) and
 *            returns 1 when the loop has ended, 0 when it stopped at that count, < 0 on
 *            error; synchronises the stream once per graph launch (32 steps by default)
 *   steps    S so far (steps with effective transformations)
 *   finish   SIGMA := diag(A), A's diagonal zeroed, Z := J Z^T J (J Z^H J); returns
 *            INFO as DSTEP_LOOP: S when the loop ended, JK_ERR_MAX_STEPS when it stopped
 *            at opts->max_steps or was not advanced to its end, < 0 on an error
 * A solver is used by one host thread at a time. */
typedef struct jk_solver jk_solver;
jk_solver *jk_solver_create(int n, int complex_, const int *J, int n_2, int id_ncp, int id_tru, const jk_opts *opts,
                            int *info);
void jk_solver_destroy(jk_solver *s);
int jk_solver_begin(jk_solver *s, double *dU, double *dA, double *dZ, void *stream);
int jk_solver_resume(jk_solver *s, double *dU, double *dA, double *dZ, const double *dsigma, long long steps,
                     void *stream);
int jk_solver_advance(jk_solver *s, long long steps);
long long jk_solver_steps(const jk_solver *s);
int jk_solver_finish(jk_solver *s, double *dsigma);

/* A batch of independent 2x2 HSVDs on the device (DHSVD2 src/D/dtransf.F90:614,
 * ZHSVD2 src/Z/ztransf.F90:925; the dtest/ztest kernel).  Host arrays: A, U, Z hold
 * `count` column-major 2x2 blocks (4 reals or 4 complex each), J 2 signs per block;
 * A is overwritten as DHSVD2 leaves it. */
int jk_dhsvd2_batch(int count, double *A, const int *J, double *U, double *Z, int *info, double th1);
int jk_zhsvd2_batch(int count, double *A, const int *J, double *U, double *Z, int *info, double th1);

/* One build's pair weights (DMAGF2T/DMAGF2H, src/D/dstep.F90:189-219; ZMAGF2T/ZMAGF2H,
 * src/Z/zstep.F90:191-221) on the device, returned as a symmetric n x n host matrix W
 * (W[p + q*n] = weight of the pair (p, q), NaN where the reference stores a NaN). */
int jk_dweights(int n, const double *A, int lda, const int *J, double *W);
int jk_zweights(int n, const double *A, int lda, const int *J, double *W);

/* The greedy non-colliding selection of one step (AW_SRT1/2 + AW_NCP1/2,
 * src/shared/atypes.F90:85-484) on the device, from a symmetric n x n host weight
 * matrix; writes SL pivots (1-based p < q) in selection order and returns SL. */
int jk_select(int n, const double *W, int n_2, int *piv);

/* A reusable device workspace for one order N and sign vector J (kernel-level use). */
typedef struct jk_handle jk_handle;
jk_handle *jk_handle_create(int n, int complex_, const int *J, int *info);
void jk_handle_destroy(jk_handle *h);

/* Enqueue one build's pair weights (the two weight kernels) of the device matrix dA
 * (leading dimension n) on `stream`; when dW is not NULL, also copy the symmetric
 * n x n weight matrix there (device pointer).  Returns 0 or an INFO error. */
int jk_handle_weights(jk_handle *h, const double *dA, double *dW, void *stream);

/* The pair weights of jk_handle_weights with no device allocation at all; no counterpart
 * in the reference.  For callers that may not allocate where they need the weights:
 * cudaMalloc/cudaFree synchronise the whole device (stalling the caller's other streams
 * in a latency-bound loop) and fail once the device memory belongs to the caller's own
 * pool.  dA (leading dimension n) and dW (n x n, only off-diagonal entries written) are
 * device pointers, J the host sign vector, stream a cudaStream_t (NULL = default).
 * Scratch (the stop flag, J and the +/- index lists) is a static device array for
 * N <= JK_NOALLOC_MAX_N; larger N returns JK_ERR_SCRATCH.  The first call on each
 * device looks up the array's device address (cudaGetSymbolAddress) and should come
 * before any stream capture on that device.  All calls on a device share the array, so
 * calls whose kernels may overlap (unordered streams) race: order them.  J is staged
 * through a pageable copy, so the call returns before the kernels finish.
 * Returns 0, -1 (N < 3), -2 (dA NULL), -4 (dW NULL), -8 (J NULL), JK_ERR_J,
 * JK_ERR_SCRATCH or a CUDA error. */
#define JK_NOALLOC_MAX_N 1024
int jk_dweights_noalloc(int n, const double *dA, const int *J, double *dW, void *stream);

/* Batched solve: `count` independent real matrices of orders n[m] (3 <= n[m] <=
 * JK_BATCH_MAX_N), each through the whole DSTEP_LOOP (src/D/dstep.F90:472-604) with its
 * own N_2 n_2[m] (clamped as JSTEP_LEN does), all in one persistent launch (one thread
 * block per matrix at a time, largest matrices first).  Packed layout: matrix m's
 * column-major n[m] x n[m] blocks of A, U, Z start at sum_{k<m} n[k]^2 doubles; its J
 * and SIGMA entries at sum_{k<m} n[k].  info[m] is the matrix's INFO (>= 0 steps, < 0
 * error).  Results equal jk_dstep_loop's on each matrix. */
#define JK_BATCH_MAX_N 128
/* The batched solver's step bound per matrix when opts->max_steps is 0: 4000 N_max + 100000
 * (N_max the batch's largest order).  The reference loop has no bound, but some inputs
 * practically never end: 7 of the 4096 matrices of the benchmark's batch (N in [16, 128])
 * were still transforming after 2e7 steps, which keeps one SM busy for 14 minutes, and one
 * persistent launch holds every matrix's results until its slowest matrix ends.  A matrix
 * that reaches the bound returns INFO JK_ERR_MAX_STEPS with A, U, Z, SIGMA as its loop
 * left them; jk_solver_resume continues it on the single-matrix loop, which has no bound. */
#define JK_BATCH_STEP_BOUND(nmax) (4000LL * (nmax) + 100000LL)
typedef struct jk_batch jk_batch;
/* A plan for one batch shape (orders, N_2, J: host arrays); opts: max_steps (0: the bound
 * above), device. */
jk_batch *jk_batch_create(int count, const int *n, const int *n_2, const int *J, const jk_opts *opts, int *info);
void jk_batch_destroy(jk_batch *b);
/* Enqueue the solve on device buffers (packed as above) on `stream`; A in/out, U, Z,
 * SIGMA, INFO out.  The launch is captured once per set of buffers as a CUDA graph
 * and replayed.  Returns 0 or an error; does not synchronise. */
int jk_batch_run(jk_batch *b, double *dA, double *dU, double *dZ, double *dsigma, int *dinfo, void *stream);
/* Autotune the block shape (threads per block) on this batch: times every candidate on
 * a copy of the batch's largest matrices (two per resident block, at most 30 N steps
 * each), keeps the fastest for later runs and returns its thread count.  dA is left
 * unchanged; dU, dZ, dsigma, dinfo are overwritten (scratch). */
int jk_batch_tune(jk_batch *b, const double *dA, double *dU, double *dZ, double *dsigma, int *dinfo, void *stream);
/* Rank the batch's scanned hyperbolic pairs by the Gram form of their weights (a scorer
 * made by jk_scorer_create with nf = 0; see the learned ranking below), with the same
 * fallback to the exact weights; sc NULL: the exact weights (the default).  Later runs and
 * tunes use it.  Returns 0, -1 (b NULL) or -2 (a scorer with a network: the batched kernel
 * has no room for one in shared memory). */
typedef struct jk_scorer jk_scorer;
int jk_batch_set_scorer(jk_batch *b, const jk_scorer *sc);
/* The same with host buffers (copies in and out, synchronous).  Returns 0 or an error. */
int jk_dstep_loop_batched(int count, const int *n, const int *n_2, double *A, double *U, double *Z, const int *J,
                          double *sigma, int *info, const jk_opts *opts);

/* The learned ranking (no counterpart in the reference, which ranks by the exact weights
 * of DMAGF2H, src/D/dstep.F90:41-72).  In a scored step the hyperbolic pairs that need the
 * O(N) column scan of ABODNDF2 (src/D/dtransf.F90:246-348) are ranked by
 *   w_gram  the same off-norm reduction written through the Gram matrix of the columns
 *           without their diagonal (one FP64 matrix product per step on the FP64 tensor
 *           pipe) and the pair's exact 2x2 transformation; it equals the exact weight up
 *           to rounding, and
 *   w       = w_gram * 2^(clamp(y, -1, 1) / 8), y the output of a network
 *           8 -> 64 -> 64 -> 1 (ReLU, BF16 weights and inputs, FP32 biases and
 *           accumulation, on the tensor cores) that learns the correction from
 *           features: log2/64 of |w_gram|, the two columns' squared off-norms without rows
 *           p, q, |their product|, |the two leading terms|, |Z12| + |Z21|; sign(w_gram);
 *           min(S / (10 N), 4).  Training target: clamp(8 log2(w / w_gram), -1, 1) with w the
 *           exact weight (0 when the signs differ).
 * The NaN tests, the other weights, the selection, the 2x2 HSVDs and the rotations stay
 * exact.  Only a step ranked by the exact weights can end the loop (a scored step without
 * an effective pivot is followed by an exact step), a step whose off-norm has not reached
 * a new minimum for `stall_k` steps is followed by an exact step, and once the off-norm
 * exceeds 16 times its minimum the rest of the solve ranks exactly.
 * Parameters (floats, FP32 master copy): W1 [64][8] (row-major), b1 [64], W2 [64][64],
 * b2 [64], W3 [64], b3: jk_mlp_nparams(8) = 4801 floats.  jk_scorer_create with nf = 0 and
 * params NULL ranks by w_gram alone (no network). */
#define JK_MLP_FEATURES 8
int jk_mlp_nparams(int nf);
jk_scorer *jk_scorer_create(int nf, const float *params, int stall_k, int *info);
void jk_scorer_destroy(jk_scorer *sc);
/* jk_dstep_loop_dev with the scored ranking; *exact_steps (optional) receives the steps
 * that ranked by the exact weights. */
int jk_dstep_loop_dev_scored(int n, double *dU, double *dA, double *dZ, const int *J, double *dsigma, int n_2,
                             const jk_scorer *sc, const jk_opts *opts, jk_trace *trace, int *exact_steps, void *stream);
/* jk_zstep_loop_dev with the scored ranking (the complex weights of ZMAGF2H,
 * src/Z/zstep.F90:43-74, whose scan ABODNZF2 sums |.|^2 of the complex entries): w_gram is
 *   d + nx (1 - |Z11|^2 - |Z12|^2) + ny (1 - |Z21|^2 - |Z22|^2)
 *     - 2 Re((conj(Z11) Z21 + conj(Z12) Z22) g),  g = x^H y,
 * the real and imaginary parts of every x^H y from the same FP64 matrix product over the
 * interleaved (re, im) columns; the network and its features are the real path's, with
 * |g| for the product. */
int jk_zstep_loop_dev_scored(int n, double *dU, double *dA, double *dZ, const int *J, double *dsigma, int n_2,
                             const jk_scorer *sc, const jk_opts *opts, jk_trace *trace, int *exact_steps, void *stream);
/* Training on the device.  jk_mlp_features writes the features of every hyperbolic pair
 * of the device matrix dA (step S = `step`) in (+ index, - index) order, the indices
 * ascending within each sign class, and returns their count; dWg (optional) receives each
 * pair's w_gram, NaN for the pairs that need no column scan (their features are zero).
 * jk_mlp_forward: the network (the inference arithmetic) on `count` feature rows.
 * jk_mlp_grad: mean squared error against dT and its gradient with respect to the FP32
 * parameters (weights used rounded to BF16), summed in a fixed order; dWork holds
 * jk_mlp_grad_workspace(nf, count) floats.  jk_mlp_adam: one Adam update of the
 * parameters (step t >= 1). */
long long jk_mlp_features(int n, const double *dA, const int *J, int step, float *dX, double *dWg, void *stream);
/* jk_mlp_features of a complex device matrix (dA: N x N double complex, column-major). */
long long jk_zmlp_features(int n, const double *dA, const int *J, int step, float *dX, double *dWg, void *stream);
int jk_mlp_forward(int nf, int count, const float *dX, const float *dParams, float *dY, void *stream);
long long jk_mlp_grad_workspace(int nf, int count);
int jk_mlp_grad(int nf, int count, const float *dX, const float *dT, const float *dParams, float *dGrad, float *dLoss,
                float *dWork, void *stream);
int jk_mlp_adam(int np, float *dParams, const float *dGrad, float *dM, float *dV, int t, float lr, float beta1,
                float beta2, float eps, void *stream);

/* Kernel launches enqueued by the calling thread's last step-loop call. */
long long jk_last_launch_count(void);

/* FP64 FMA throughput of the current device in TFLOP/s (2 flops per fma), from a
 * dependent-chain kernel with 8 chains per thread over a full grid; the peak the
 * FP64 roofline is quoted against. */
double jk_fp64_peak(void);

/* Largest order N the loops accept. */
int jk_max_order(int complex_);

/* Text for an INFO code. */
const char *jk_strerror(int info);

#ifdef __cplusplus
}
#endif
#endif /* !JKOGB_H */
