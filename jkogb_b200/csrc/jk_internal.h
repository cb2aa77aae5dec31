// jk_internal.h -- device data layout and host launch wrappers shared by the
// CUDA translation units of libjkogb_b200 (not part of the public C ABI).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace jk {

// Loop state kept on the device (one per solve).  Mirrors the scalars of
// DSTEP_LOOP / DSTEP_EXEC (src/D/dstep.F90:376-604).
struct State {
  int stop;    // 1 once the loop has ended; 2 while it waits at `limit` (resumable)
  int steps;   // S: steps with effective transformations
  int info;    // final INFO (valid once stop)
  int sl;      // SL of the current step (selected pivots)
  int nl;      // NL: effective pivots of the current step
  int err;     // minimum negative INFO over the current step's pivots (0 if none)
  int nunp;    // columns outside the current pivot set
  int rounds;  // matching rounds of the current step
  int pending; // a step whose end-of-step test is still to run
  int trace_on;
  int trace_steps;      // steps recorded in the trace
  int trace_cap_steps;  // capacity (steps) of the trace arrays
  long long trace_npiv; // pivots recorded
  long long trace_cap_piv;
  double tw;   // sum of the weights of the effective pivots (NORMF2D column)
  int trig, hyp;
  // the learned ranking (jk_scorer): off unless `learned`
  int learned;       // the solve ranks the scanned hyperbolic pairs by the scorer
  int learned_step;  // this step uses the scorer (0: the exact weights)
  int stall;         // steps since the off-norm last reached a new minimum
  int stall_k;       // after this many such steps the next step is exact
  int exact_steps;   // steps run with the exact weights in a learned solve
  int retry;         // a learned step without an effective pivot: the loop goes on with an exact step
  double off, best_off;  // off-norm after the last step, its minimum so far
  long long limit;   // the loop waits (stop = 2) once `steps` reaches this (0: never)
};

// Per-step trace on the device (optional).
struct Trace {
  int *sl, *nl, *trig, *hyp, *rounds;
  double *tw;
  int2 *piv;  // 0-based (p, q)
};

// One selected pivot (rank order) and its 2x2 transformation.
template <typename T>
struct Piv {
  int p, q, info, pad;
  double w;       // its weight (for the statistics)
  T V[4];         // left 2x2 of DHSVD2 (before UT2/UH2)
  T W[4];         // right 2x2 (Z of DHSVD2), W(:,1:2,I) of DSTEP_TRANSF
  double d[2];    // W(1,3,I), W(2,3,I): the new diagonal
};

// Row-rotation record of one pivot: the BA coefficients of V (read by every block).
template <typename T>
struct RowRot {
  int p, q, flags, pad;  // flags: bit0 c1, bit1 c2, bit2 apply
  T r1, r2, m1, m2;
};

// scan parameters of one hyperbolic pair (real path)
struct HypPar {
  double r1, r2, m1, m2, d;  // the AB coefficients of Z2 and the two leading terms
  int p, q;                  // the pair (0-based, p < q)
  int flags;                 // bit0 scan, bit1 c1, bit2 c2
  int pad;
};

// the scorer of a learned solve (device parameters)
struct ScorerDev {
  const unsigned short *w;  // bf16 weights W1 [64][nf], W2 [64][64], W3 [64] (NULL: no network)
  const float *b;           // fp32 biases b1 [64], b2 [64], b3
  int nf;
};

struct Workspace {
  int n;
  int cplx;
  int n_plus, n_minus;
  int *J;            // signs (device)
  int *plus, *minus; // indices with J=+1 / J=-1, ascending
  double *Wm;        // n x n pair weights, symmetric, NaN = no transformation
  double *mag;       // complex: n x n magnitudes |A(i,j)| of the step
  void *piv;         // Piv<T>[n/2]
  void *rowrot;      // RowRot<T>[n/2]
  unsigned short *list;  // n x list_ld(n): the partners of every vertex, best first
  unsigned short *rank;  // n x n: rank[v][u] = position of u in v's list
  int *len;              // valid entries of each list
  int *unp;              // columns outside the current pivot set
  State *st;         // device state
  State *st_host;    // pinned host mirror
  Trace tr;
  int zba_quirk;
  double *offpart;   // per-block partial off-norms (learned solves)
  int *offcount;     // blocks done (the last one finishes the off-norm)
  int learned;       // rank the scanned hyperbolic pairs by `sc`
  ScorerDev sc;      // sc.nf == 0: the Gram form alone (no network)
  double *gram;      // scored steps: n_plus x n_minus products of the columns without their diagonal
  double *cn;        // ... and the columns' off-diagonal squared norms
  // ID_NCP = 3 (AW_NCP3): per record key and tie, the sorted order, every start's walk
  int id_ncp;
  unsigned long long *n3key;
  unsigned *n3tie;
  int *n3sorted, *n3len, *n3it;
  double *n3val;
};
constexpr int kNcp3MaxN = 256;  // AW_NCP3's work grows as the square of the record count

// host launchers (jk_kernels.cu)
cudaError_t launch_init(Workspace &w, void *U, void *Z, int learned, int stall_k, int steps0, int fresh, cudaStream_t s);
cudaError_t launch_unfinish(Workspace &w, void *A, void *Z, const double *sigma, cudaStream_t s);
cudaError_t launch_limit(Workspace &w, long long limit, cudaStream_t s);
cudaError_t launch_step(Workspace &w, void *A, void *U, void *Z, int n_2, cudaStream_t s);
cudaError_t launch_finish(Workspace &w, void *A, void *Z, double *sigma, cudaStream_t s);
cudaError_t launch_weights(Workspace &w, const void *A, cudaStream_t s);
cudaError_t launch_match(Workspace &w, int n_2, cudaStream_t s);
cudaError_t launch_hsvd2_batch(int cplx, int count, void *A, const int *J, void *U, void *Z, int *info, double th1, cudaStream_t s);
cudaError_t prepare_kernels(int n);
// the batched solver (jk_batch.cu): one matrix of the packed batch
struct BatchItem {
  long long off;  // offset of its n x n blocks in A, U, Z (doubles)
  int n, n_2;     // order and N_2 (clamped as JSTEP_LEN does)
  int joff;       // offset of its J and SIGMA entries
  int index;      // position in the caller's batch (INFO slot)
};
constexpr int kBatchMaxN = 128;
constexpr int kBatchVariants = 3;
constexpr int kInfoMaxSteps = -24;
constexpr int kInfoSelect = -25;  // the batched selection exceeded its iteration bound (internal error)
extern const int kBatchThreads[kBatchVariants];
size_t batch_smem(int nm);
cudaError_t batch_prepare(int nm);
int batch_blocks_per_sm(int variant, int nm);
cudaError_t launch_batch(int variant, int grid, const BatchItem *items, int count, int *counter, double *A, double *U,
                         double *Z, const int *J, double *sigma, int *info, int nm, long long cap, int scored, int stall_k,
                         cudaStream_t s);

// the learned ranking (jk_scorer.cu)
constexpr int kMlpHidden = 64;
constexpr int kMlpFeat = 8;
__host__ __device__ constexpr int mlp_params(int nf) { return kMlpHidden * nf + kMlpHidden + kMlpHidden * kMlpHidden + kMlpHidden + kMlpHidden + 1; }
cudaError_t launch_learned_weights(Workspace &w, const void *A, cudaStream_t s);
cudaError_t prepare_gram();
constexpr int kOffBlocks = 296;  // fixed grid of the off-norm reduction (a fixed summation order)
cudaError_t launch_offnorm(Workspace &w, const void *A, cudaStream_t s);
cudaError_t mlp_features(int cplx, int n, const void *A, const int *plus, const int *minus, int n_plus, int n_minus,
                         int step, const State *st, double *G, double *cn, float *X, double *Wg, cudaStream_t s);
cudaError_t mlp_forward(int nf, int count, const float *X, const unsigned short *w, const float *b, float *Y, cudaStream_t s);
cudaError_t mlp_grad(int nf, int count, const float *X, const float *T, const float *params, float *grad, float *loss,
                     float *partial, cudaStream_t s);
size_t mlp_grad_partial_floats(int nf, int count);
cudaError_t mlp_adam(int np, float *params, const float *grad, float *m, float *v, int t, float lr, float b1, float b2,
                     float eps, cudaStream_t s);
cudaError_t mlp_pack(int nf, const float *params, unsigned short *w, float *b, cudaStream_t s);

// weights of a real matrix with no allocation: scratch in a static device array
constexpr int kNoallocMaxN = 1024;
cudaError_t launch_weights_noalloc(int n, const double *A, const int *J, double *W, cudaStream_t s);
double fp64_peak();
// kernel launches of one step (the graph body)
constexpr int kStepLaunches = 6;
size_t select_smem(int n);
int colsort_e(int n);

}  // namespace jk
