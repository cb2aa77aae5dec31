// jk_scorer.cu -- the learned ranking of the hyperbolic pairs: a small MLP that
// predicts a pair's weight (its off-norm reduction, DMAGF2H src/D/dstep.F90:41-72)
// from the pair's own 2x2 block, so that a step can rank the pairs without the O(N)
// column scan of ABODNDF2 (src/D/dtransf.F90:246-348) per pair.  It replaces the
// weight only for ranking: the "no transformation" tests (NaN), the weights that
// need no scan, the selection, the 2x2 HSVDs, the rotations and the end-of-loop
// test stay exact.  When the off-norm has not reached a new minimum for `stall_k`
// steps, the next step ranks by the exact weights.
//
// Network: 7 features -> 64 (ReLU) -> 64 (ReLU) -> 1, BF16 weights, FP32 biases and
// FP32 accumulation.  Features of the pair p < q (A(i,j) at that step):
//   log2|A(p,q)|/64, log2|A(q,p)|/64, log2|A(p,p)|/64, log2|A(q,q)|/64 (zero counts as
//   2^-1074), J(p), J(q), min(S / (10 N), 4) with S the steps so far.
// Target: the exact weight w through g(w) = sign(w) (log2|w| + 1100) / 1024 (g(0) = 0),
// a monotone map in which the sign dominates the error, so that ranking by the
// prediction ranks by the predicted weight; the prediction enters the record list as
// g^-1 of it.  (A map that spreads the magnitudes more, log2(1 + 2^80 |w|) / 16, let
// the scorer pick off-norm-raising hyperbolic pairs often enough for the entries to
// grow without bound.)
//
// Also here: the training kernels (forward, backward into per-block partial
// gradients reduced in a fixed order, Adam) and the per-step off-norm.
#include <cuda_bf16.h>

#include "jk_internal.h"
#include "jk_device.cuh"

namespace jk {

namespace {

constexpr int H = kMlpHidden;
constexpr int NF = kMlpFeat;

// parameter layout (floats): W1 [H][NF], b1 [H], W2 [H][H], b2 [H], W3 [H], b3
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + H * NF, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H, OFF_W3 = OFF_B2 + H,
              OFF_B3 = OFF_W3 + H, NPARAM = OFF_B3 + 1;
static_assert(NPARAM == mlp_params(NF), "parameter layout");

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float bf16_load(unsigned short u) { return __bfloat162float(__ushort_as_bfloat16(u)); }

__device__ __forceinline__ float lg64(double x)
{
  const double a = fabs(x);
  return (float)(((a > 0.0) ? log2(a) : -1074.0) * (1.0 / 64.0));
}

// the features of pair p < q
__device__ __forceinline__ void pair_features(double app, double aqp, double apq, double aqq, int jp, int jq, int step, int n,
                                              float x[NF])
{
  x[0] = lg64(apq);
  x[1] = lg64(aqp);
  x[2] = lg64(app);
  x[3] = lg64(aqq);
  x[4] = (float)jp;
  x[5] = (float)jq;
  x[6] = fminf((float)step / (10.0f * (float)n), 4.0f);
}

// g^-1 of a prediction: the weight it stands for in the record order
__device__ __forceinline__ double g_inverse(float y)
{
  const double e = fabs((double)y) * 1024.0 - 1100.0;
  const double m = exp2(e < -1100.0 ? -1100.0 : (e > 1100.0 ? 1100.0 : e));
  return (y < 0.0f) ? -m : m;
}

// the network in shared memory (FP32 copies of the BF16 weights)
struct SNet {
  float w1[H * NF], b1[H], w2[H * H], b2[H], w3[H], b3;
};

__device__ void load_net_packed(SNet &s, const ScorerDev &sc)
{
  for (int k = threadIdx.x; k < H * NF; k += blockDim.x) s.w1[k] = bf16_load(sc.w[k]);
  for (int k = threadIdx.x; k < H * H; k += blockDim.x) s.w2[k] = bf16_load(sc.w[H * NF + k]);
  for (int k = threadIdx.x; k < H; k += blockDim.x) {
    s.w3[k] = bf16_load(sc.w[H * NF + H * H + k]);
    s.b1[k] = sc.b[k];
    s.b2[k] = sc.b[H + k];
  }
  if (threadIdx.x == 0) s.b3 = sc.b[2 * H];
}

// from FP32 master parameters, rounded to BF16 as inference sees them
__device__ void load_net_master(SNet &s, const float *P)
{
  for (int k = threadIdx.x; k < H * NF; k += blockDim.x) s.w1[k] = bf16_round(P[OFF_W1 + k]);
  for (int k = threadIdx.x; k < H * H; k += blockDim.x) s.w2[k] = bf16_round(P[OFF_W2 + k]);
  for (int k = threadIdx.x; k < H; k += blockDim.x) {
    s.w3[k] = bf16_round(P[OFF_W3 + k]);
    s.b1[k] = P[OFF_B1 + k];
    s.b2[k] = P[OFF_B2 + k];
  }
  if (threadIdx.x == 0) s.b3 = P[OFF_B3];
}

// forward pass of one sample, FP32 accumulation in a fixed order
__device__ __forceinline__ float net_forward(const SNet &s, const float x[NF])
{
  float h1[H];
#pragma unroll
  for (int j = 0; j < H; ++j) {
    float a = s.b1[j];
#pragma unroll
    for (int f = 0; f < NF; ++f) a = fmaf(s.w1[j * NF + f], x[f], a);
    h1[j] = fmaxf(a, 0.0f);
  }
  float y = s.b3;
  for (int j = 0; j < H; ++j) {
    float a = s.b2[j];
#pragma unroll
    for (int i = 0; i < H; ++i) a = fmaf(s.w2[j * H + i], h1[i], a);
    y = fmaf(s.w3[j], fmaxf(a, 0.0f), y);
  }
  return y;
}

// ---------------------------------------------------------------------------
// the weights of the hyperbolic pairs in a learned step: DMAGF2H's 2x2 part exact;
// a pair that needs the column scan is scored by the network instead
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k_hyp_learned(const State *st, const double *__restrict__ A, const int *__restrict__ plus, const int *__restrict__ minus,
              int n_plus, int n_minus, double *__restrict__ Wm, int n, ScorerDev sc)
{
  if (st->stop || !st->learned_step) return;
  __shared__ SNet net;
  load_net_packed(net, sc);
  __syncthreads();
  const int ia = blockIdx.x * 16 + (threadIdx.x & 15), ib = blockIdx.y * 16 + (threadIdx.x >> 4);
  if (ia >= n_plus || ib >= n_minus) return;
  const int a = plus[ia], b = minus[ib];
  const bool a_is_p = a < b;
  const int p = a_is_p ? a : b, q = a_is_p ? b : a;
  const double app = A[(long long)p * n + p], aqp = A[(long long)p * n + q], apq = A[(long long)q * n + p],
               aqq = A[(long long)q * n + q];
  double w, d;
  Rot t;
  if (hyp_setup(app, aqp, apq, aqq, a_is_p ? 1 : -1, w, d, t)) {
    float x[NF];
    pair_features(app, aqp, apq, aqq, a_is_p ? 1 : -1, a_is_p ? -1 : 1, st->steps, n, x);
    w = g_inverse(net_forward(net, x));
  }
  if (w < -JK_HUGE) w = nan_w();
  Wm[(long long)q * n + p] = w;
  Wm[(long long)p * n + q] = w;
}

// the off-norm sum_{i != j} A(i,j)^2 after a learned step, in a fixed summation order
// (per-block tree sums, then the last block adds the block sums in block order), and
// the choice of the next step's ranking
__global__ void __launch_bounds__(256)
k_offnorm(State *st, const double *__restrict__ A, int n, double *part, int *count)
{
  if (st->stop || !st->learned) return;
  __shared__ double red[256];
  __shared__ int last;
  const long long nn = (long long)n * n;
  double acc = 0.0;
  for (long long k = blockIdx.x * 256LL + threadIdx.x; k < nn; k += (long long)gridDim.x * 256) {
    const int i = (int)(k % n), j = (int)(k / n);
    if (i != j) acc = fma(A[k], A[k], acc);
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[blockIdx.x] = red[0];
    __threadfence();
    last = (atomicAdd(count, 1) == (int)gridDim.x - 1);
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  double off = 0.0;
  for (int b = 0; b < (int)gridDim.x; ++b) off += ((volatile double *)part)[b];
  *count = 0;
  st->off = off;
  const int sl = st->sl, nl = st->nl;
  if (st->learned_step && st->err == 0 && ((sl < nl) ? sl : nl) <= 0) {
    // no effective pivot among the learned choices: the end-of-loop test is left to an
    // exact step
    st->retry = 1;
    st->learned_step = 0;
    st->stall = 0;
    st->exact_steps += 1;
    return;
  }
  if (off > 16.0 * st->best_off) {
    // the learned choices let the off-norm grow: the rest of the solve ranks exactly
    st->learned = 0;
    st->learned_step = 0;
    st->exact_steps += 1;
    return;
  }
  if (off < st->best_off) { st->best_off = off; st->stall = 0; }
  else st->stall += 1;
  if (st->stall >= st->stall_k) {
    st->learned_step = 0;  // the next step ranks by the exact weights
    st->stall = 0;
    st->exact_steps += 1;
  }
  else
    st->learned_step = 1;
}

// ---------------------------------------------------------------------------
// training data and training
// ---------------------------------------------------------------------------
// features of every hyperbolic pair in (+ index, - index) order: X [n_plus * n_minus][NF]
__global__ void k_features(const double *__restrict__ A, const int *__restrict__ plus, const int *__restrict__ minus,
                           int n_plus, int n_minus, int n, int step, float *X)
{
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= (long long)n_plus * n_minus) return;
  const int a = plus[k / n_minus], b = minus[k % n_minus];
  const bool a_is_p = a < b;
  const int p = a_is_p ? a : b, q = a_is_p ? b : a;
  float x[NF];
  pair_features(A[(long long)p * n + p], A[(long long)p * n + q], A[(long long)q * n + p], A[(long long)q * n + q],
                a_is_p ? 1 : -1, a_is_p ? -1 : 1, step, n, x);
#pragma unroll
  for (int f = 0; f < NF; ++f) X[k * NF + f] = x[f];
}

__global__ void __launch_bounds__(128)
k_mlp_forward(const float *__restrict__ X, const float *__restrict__ P, int count, float *Y)
{
  __shared__ SNet net;
  load_net_master(net, P);
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= count) return;
  float x[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) x[f] = X[(long long)s * NF + f];
  Y[s] = net_forward(net, x);
}

constexpr int GB = 128;  // samples per block of the gradient kernel

// loss = mean (y - t)^2 over `count` samples; this block's partial gradient (and
// loss) of its GB samples into part[blockIdx.x][NPARAM + 1]
__global__ void __launch_bounds__(GB)
k_mlp_grad(const float *__restrict__ X, const float *__restrict__ T, const float *__restrict__ P, int count, float *part)
{
  __shared__ SNet net;
  extern __shared__ float dyn[];
  float *h1 = dyn;               // [GB][H] activations, later their gradients
  float *h2 = h1 + GB * H;       // [GB][H] activations, later their gradients
  float *xs = h2 + GB * H;       // [GB][NF]
  float *dy = xs + GB * NF;      // [GB]
  load_net_master(net, P);
  const int tid = threadIdx.x, s = blockIdx.x * GB + tid;
  const bool valid = s < count;
  const float inv = 1.0f / (float)count;
  float x[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) { x[f] = valid ? X[(long long)s * NF + f] : 0.0f; xs[tid * NF + f] = x[f]; }
  __syncthreads();
  // forward, keeping the activations
  float y = net.b3;
  for (int j = 0; j < H; ++j) {
    float a = net.b1[j];
#pragma unroll
    for (int f = 0; f < NF; ++f) a = fmaf(net.w1[j * NF + f], x[f], a);
    h1[tid * H + j] = fmaxf(a, 0.0f);
  }
  for (int j = 0; j < H; ++j) {
    float a = net.b2[j];
    for (int i = 0; i < H; ++i) a = fmaf(net.w2[j * H + i], h1[tid * H + i], a);
    a = fmaxf(a, 0.0f);
    h2[tid * H + j] = a;
    y = fmaf(net.w3[j], a, y);
  }
  const float r = valid ? (y - T[s]) : 0.0f;
  dy[tid] = 2.0f * r * inv;
  float *out = part + (long long)blockIdx.x * (NPARAM + 1);
  __syncthreads();
  // dW3, db3, the loss
  for (int j = tid; j < H; j += GB) {
    float g = 0.0f;
    for (int t = 0; t < GB; ++t) g = fmaf(dy[t], h2[t * H + j], g);
    out[OFF_W3 + j] = g;
  }
  if (tid == 0) {
    float g = 0.0f;
    for (int t = 0; t < GB; ++t) g += dy[t];
    out[OFF_B3] = g;
  }
  __syncthreads();
  // dh2 = dy W3 (h2 > 0), in place
  for (int j = 0; j < H; ++j) {
    const float a = h2[tid * H + j];
    h2[tid * H + j] = (a > 0.0f) ? dy[tid] * net.w3[j] : 0.0f;
  }
  __syncthreads();
  // dW2 [j][i] = sum_t dh2[t][j] h1[t][i]; db2
  for (int e = tid; e < H * H; e += GB) {
    const int j = e / H, i = e % H;
    float g = 0.0f;
    for (int t = 0; t < GB; ++t) g = fmaf(h2[t * H + j], h1[t * H + i], g);
    out[OFF_W2 + e] = g;
  }
  for (int j = tid; j < H; j += GB) {
    float g = 0.0f;
    for (int t = 0; t < GB; ++t) g += h2[t * H + j];
    out[OFF_B2 + j] = g;
  }
  __syncthreads();
  // dh1 = W2^T dh2 (h1 > 0), in place (own row only)
  {
    float d1[H];
#pragma unroll
    for (int i = 0; i < H; ++i) d1[i] = 0.0f;
    for (int j = 0; j < H; ++j) {
      const float g = h2[tid * H + j];
#pragma unroll
      for (int i = 0; i < H; ++i) d1[i] = fmaf(net.w2[j * H + i], g, d1[i]);
    }
#pragma unroll
    for (int i = 0; i < H; ++i) h1[tid * H + i] = (h1[tid * H + i] > 0.0f) ? d1[i] : 0.0f;
  }
  __syncthreads();
  // dW1 [i][f], db1
  for (int e = tid; e < H * NF; e += GB) {
    const int i = e / NF, f = e % NF;
    float g = 0.0f;
    for (int t = 0; t < GB; ++t) g = fmaf(h1[t * H + i], xs[t * NF + f], g);
    out[OFF_W1 + e] = g;
  }
  for (int i = tid; i < H; i += GB) {
    float g = 0.0f;
    for (int t = 0; t < GB; ++t) g += h1[t * H + i];
    out[OFF_B1 + i] = g;
  }
  // this block's share of the loss
  __syncthreads();
  dy[tid] = r * r * inv;
  __syncthreads();
  if (tid == 0) {
    float l = 0.0f;
    for (int t = 0; t < GB; ++t) l += dy[t];
    out[NPARAM] = l;
  }
}

// grad[k] = sum over blocks of part[b][k], in block order (k = NPARAM: the loss)
__global__ void k_mlp_reduce(const float *__restrict__ part, int blocks, float *grad, float *loss)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k > NPARAM) return;
  float g = 0.0f;
  for (int b = 0; b < blocks; ++b) g += part[(long long)b * (NPARAM + 1) + k];
  if (k < NPARAM) grad[k] = g;
  else *loss = g;
}

__global__ void k_mlp_adam(int np, float *P, const float *__restrict__ G, float *M, float *V, float lr, float b1, float b2,
                           float eps, float c1, float c2)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= np) return;
  const float g = G[k];
  const float m = b1 * M[k] + (1.0f - b1) * g;
  const float v = b2 * V[k] + (1.0f - b2) * g * g;
  M[k] = m;
  V[k] = v;
  P[k] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

// FP32 master parameters -> the inference form (BF16 weights, FP32 biases)
__global__ void k_mlp_pack(const float *__restrict__ P, unsigned short *w, float *b)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < H * NF) w[k] = __bfloat16_as_ushort(__float2bfloat16_rn(P[OFF_W1 + k]));
  if (k < H * H) w[H * NF + k] = __bfloat16_as_ushort(__float2bfloat16_rn(P[OFF_W2 + k]));
  if (k < H) {
    w[H * NF + H * H + k] = __bfloat16_as_ushort(__float2bfloat16_rn(P[OFF_W3 + k]));
    b[k] = P[OFF_B1 + k];
    b[H + k] = P[OFF_B2 + k];
  }
  if (k == 0) b[2 * H] = P[OFF_B3];
}

}  // namespace

cudaError_t launch_gram_weights(Workspace &w, const double *A, cudaStream_t s);

cudaError_t launch_learned_weights(Workspace &w, const double *A, cudaStream_t s)
{
  if (w.sc.nf == 0) return launch_gram_weights(w, A, s);  // the Gram-guided ranking, no network
  if (w.n_plus > 0 && w.n_minus > 0) {
    dim3 g((w.n_plus + 15) / 16, (w.n_minus + 15) / 16);
    k_hyp_learned<<<g, 256, 0, s>>>(w.st, A, w.plus, w.minus, w.n_plus, w.n_minus, w.Wm, w.n, w.sc);
  }
  return cudaGetLastError();
}

cudaError_t launch_offnorm(Workspace &w, const double *A, cudaStream_t s)
{
  k_offnorm<<<kOffBlocks, 256, 0, s>>>(w.st, A, w.n, w.offpart, w.offcount);
  return cudaGetLastError();
}

cudaError_t mlp_features(int n, const double *A, const int *plus, const int *minus, int n_plus, int n_minus, int step, int nf,
                         float *X, cudaStream_t s)
{
  if (nf != NF) return cudaErrorInvalidValue;
  const long long cnt = (long long)n_plus * n_minus;
  if (cnt > 0) k_features<<<(unsigned)((cnt + 255) / 256), 256, 0, s>>>(A, plus, minus, n_plus, n_minus, n, step, X);
  return cudaGetLastError();
}

cudaError_t mlp_forward(int nf, int count, const float *X, const float *params, float *Y, cudaStream_t s)
{
  if (nf != NF) return cudaErrorInvalidValue;
  if (count > 0) k_mlp_forward<<<(count + 127) / 128, 128, 0, s>>>(X, params, count, Y);
  return cudaGetLastError();
}

size_t mlp_grad_partial_floats(int nf, int count)
{
  const int blocks = (count + GB - 1) / GB;
  return (size_t)blocks * (mlp_params(nf) + 1);
}

cudaError_t mlp_grad(int nf, int count, const float *X, const float *T, const float *params, float *grad, float *loss,
                     float *partial, cudaStream_t s)
{
  if (nf != NF || count <= 0) return cudaErrorInvalidValue;
  const int blocks = (count + GB - 1) / GB;
  const size_t dyn = (size_t)(2 * GB * H + GB * NF + GB) * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  if (e != cudaSuccess) return e;
  k_mlp_grad<<<blocks, GB, dyn, s>>>(X, T, params, count, partial);
  k_mlp_reduce<<<(NPARAM + 1 + 255) / 256, 256, 0, s>>>(partial, blocks, grad, loss);
  return cudaGetLastError();
}

cudaError_t mlp_adam(int np, float *params, const float *grad, float *m, float *v, int t, float lr, float b1, float b2,
                     float eps, cudaStream_t s)
{
  const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
  k_mlp_adam<<<(np + 255) / 256, 256, 0, s>>>(np, params, grad, m, v, lr, b1, b2, eps, c1, c2);
  return cudaGetLastError();
}

cudaError_t mlp_pack(int nf, const float *params, unsigned short *w, float *b, cudaStream_t s)
{
  if (nf != NF) return cudaErrorInvalidValue;
  k_mlp_pack<<<(H * H + 255) / 256, 256, 0, s>>>(params, w, b);
  return cudaGetLastError();
}

}  // namespace jk

namespace jk {

// ---------------------------------------------------------------------------
// The Gram-guided ranking.  A hyperbolic pair (p, q) that needs the column scan of
// ABODNDF2 (src/D/dtransf.F90:246-348) has the weight
//   d0 + sum_{i != p,q} (x_i^2 - x_i'^2) + (y_i^2 - y_i'^2),  x = A(:,p), y = A(:,q),
// with x_i' = Z11 x_i + Z21 y_i, y_i' = Z12 x_i + Z22 y_i (Z2 the pair's 2x2 right
// transformation).  The sum is, exactly in real arithmetic,
//   nx (1 - Z11^2 - Z12^2) + ny (1 - Z21^2 - Z22^2) - 2 (Z11 Z21 + Z12 Z22) g
// with nx = sum_{i != p,q} x_i^2, ny likewise and g = sum_{i != p,q} x_i y_i: a function of
// three entries of the Gram matrix of A with its diagonal set to zero.  All of g for the
// "+" x "-" pairs is one FP64 matrix product (k_gram, on the FP64 tensor pipe, DMMA);
// nx, ny come from the columns' off-diagonal norms.  The result differs from the
// reference's sequential sum only in rounding, so it ranks the pairs as the exact weight
// does except between near-equal weights; the selection, the 2x2 HSVDs, the rotations and
// the end-of-loop test stay exact.
// ---------------------------------------------------------------------------

// column off-diagonal norms cn[j] = sum_{i != j} A(i,j)^2 (one warp per column)
__global__ void __launch_bounds__(256)
k_colnorm(const State *st, const double *__restrict__ A, int n, double *__restrict__ cn)
{
  if (st->stop || !st->learned_step) return;
  const int lane = threadIdx.x & 31;
  for (int j = blockIdx.x * 8 + (threadIdx.x >> 5); j < n; j += gridDim.x * 8) {
    const double *c = A + (long long)j * n;
    double s = 0.0;
    for (int i = lane; i < n; i += 32)
      if (i != j) s = fma(c[i], c[i], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    if (!lane) cn[j] = s;
  }
}

// G[a][b] = sum_i A0(i, plus[a]) A0(i, minus[b]) with A0 = A minus its diagonal:
// a 64 x 64 tile per block of 4 warps (32 x 32 each, 4 x 4 DMMA m8n8k4 tiles), row
// chunks of 32 staged with cp.async in two buffers; the diagonal entries are masked
// when the fragments are read.
#define GT 64
#define GK 32
#define GKP 36  // padded chunk row: the 8 x 4 fragment reads hit distinct banks
constexpr size_t kGramOperand = 2 * GT * GKP * sizeof(double);  // one operand's two buffers

__device__ __forceinline__ void dmma_8x8x4(double (&c)[2], double a, double b)
{
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async16g(void *smem, const void *gmem, bool full)
{
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = full ? 16 : 0;  // 0: the 16 bytes are zero-filled
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(sz));
}

__global__ void __launch_bounds__(128)
k_gram(const State *st, const double *__restrict__ A, const int *__restrict__ plus, const int *__restrict__ minus,
       int n_plus, int n_minus, int n, double *__restrict__ G)
{
  if (st->stop || !st->learned_step) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double (*xs)[GT][GKP] = (double (*)[GT][GKP])smem_raw;            // [2][GT][GKP]
  double (*ys)[GT][GKP] = (double (*)[GT][GKP])(smem_raw + kGramOperand);
  __shared__ int cx[GT], cy[GT];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int a0 = blockIdx.x * GT, b0 = blockIdx.y * GT;
  if (tid < GT) {
    cx[tid] = (a0 + tid < n_plus) ? plus[a0 + tid] : -1;
    cy[tid] = (b0 + tid < n_minus) ? minus[b0 + tid] : -1;
  }
  __syncthreads();
  const int nk = (n + GK - 1) / GK;
  // staging: 2 operands x 64 columns x 16 pieces of 16 bytes (two rows each) = 2048
  // copies, 16 per thread; a piece that is not 16-byte aligned in A or runs past row n
  // is loaded by plain loads (zeros past the end)
  auto stage = [&](int c) {
    if (c < nk) {
      const int k0 = c * GK, buf = c & 1;
#pragma unroll
      for (int t = 0; t < 16; ++t) {
        const int idx = tid + 128 * t;        // 0 .. 2047
        const int op = idx >> 10, col = (idx >> 4) & 63, piece = idx & 15;
        const int g = op ? cy[col] : cx[col];
        const int r = k0 + 2 * piece;
        double *dst = op ? &ys[buf][col][2 * piece] : &xs[buf][col][2 * piece];
        const long long e = (long long)g * n + r;
        if (g >= 0 && r + 1 < n && !(e & 1)) cp_async16g(dst, A + e, true);  // 16-byte aligned piece
        else {
          dst[0] = (g >= 0 && r < n) ? A[e] : 0.0;
          dst[1] = (g >= 0 && r + 1 < n) ? A[e + 1] : 0.0;
        }
      }
    }
    asm volatile("cp.async.commit_group;\n" ::);
  };
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;  // the warp's 32 x 32 sub-tile
  const int fr = lane >> 2, fk = lane & 3;                   // fragment row / k of this lane
  int gxa[4], gyb[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) { gxa[i] = cx[wm + 8 * i + fr]; gyb[i] = cy[wn + 8 * i + fr]; }
  stage(0);
  for (int c = 0; c < nk; ++c) {
    stage(c + 1);
    asm volatile("cp.async.wait_group 1;\n" ::);
    __syncthreads();
    const int buf = c & 1, k0 = c * GK;
#pragma unroll
    for (int kk = 0; kk < GK; kk += 4) {
      const int row = k0 + kk + fk;  // the matrix row this lane's fragments hold
      double fa[4], fb[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        fa[i] = (row == gxa[i]) ? 0.0 : xs[buf][wm + 8 * i + fr][kk + fk];
        fb[i] = (row == gyb[i]) ? 0.0 : ys[buf][wn + 8 * i + fr][kk + fk];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j], fa[i], fb[j]);
    }
    __syncthreads();
  }
  asm volatile("cp.async.wait_group 0;\n" ::);
  // C fragment: row fr, columns 2 fk, 2 fk + 1 of each 8 x 8 tile
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int a = a0 + wm + 8 * i + fr;
    if (a >= n_plus) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int b = b0 + wn + 8 * j + 2 * fk;
      if (b < n_minus) G[(long long)a * n_minus + b] = acc[i][j][0];
      if (b + 1 < n_minus) G[(long long)a * n_minus + b + 1] = acc[i][j][1];
    }
  }
}


// the weights of the hyperbolic pairs of a Gram-guided step: the 2x2 part of DMAGF2H
// exact (src/D/dstep.F90:41-72), the scanned part from the Gram entries
__global__ void __launch_bounds__(256)
k_hyp_gram(const State *st, const double *__restrict__ A, const int *__restrict__ plus, const int *__restrict__ minus,
           int n_plus, int n_minus, int n, const double *__restrict__ G, const double *__restrict__ cn,
           double *__restrict__ Wm)
{
  if (st->stop || !st->learned_step) return;
  const long long k = blockIdx.x * 256LL + threadIdx.x;
  if (k >= (long long)n_plus * n_minus) return;
  const int ia = (int)(k / n_minus), ib = (int)(k % n_minus);
  const int a = plus[ia], b = minus[ib];
  const bool a_is_p = a < b;
  const int p = a_is_p ? a : b, q = a_is_p ? b : a;
  const double app = A[(long long)p * n + p], aqp = A[(long long)p * n + q], apq = A[(long long)q * n + p],
               aqq = A[(long long)q * n + q];
  double w = nan_w();
  if (may_transform(app, aqp, apq, aqq)) {
    double A2[4] = { app, aqp, apq, aqq }, U2[4], Z2[4];
    int info = 0;
    const int jp = a_is_p ? 1 : -1;
    dhsvd2(A2, jp, -jp, U2, Z2, JK_TH1FIX, info);
    if (info < 0) w = nan_w();
    else if (!(info & 1)) w = 0.0;
    else if (!(info & 4)) w = dasum2(aqp, apq);
    else {
      const double a1 = (info & 8) ? A2[M21] : 0.0, a2 = (info & 8) ? A2[M12] : 0.0;
      double d = 0.0;
      d = fma(__dsub_rn(aqp, a1), __dadd_rn(aqp, a1), d);
      d = fma(__dsub_rn(apq, a2), __dadd_rn(apq, a2), d);
      const double z11 = Z2[M11], z21 = Z2[M21], z12 = Z2[M12], z22 = Z2[M22];
      const double nx = cn[p] - aqp * aqp, ny = cn[q] - apq * apq;
      const double g = G[(long long)ia * n_minus + ib];
      // 1 - z11^2 - z12^2 and 1 - z21^2 - z22^2 without cancellation at z11, z22 near +-1
      const double c1 = (1.0 - z11) * (1.0 + z11) - z12 * z12;
      const double c2 = (1.0 - z22) * (1.0 + z22) - z21 * z21;
      const double c3 = z11 * z21 + z12 * z22;
      w = d + (nx * c1 + ny * c2 - 2.0 * c3 * g);
    }
  }
  if (w < -JK_HUGE) w = nan_w();
  Wm[(long long)q * n + p] = w;
  Wm[(long long)p * n + q] = w;
}

cudaError_t launch_gram_weights(Workspace &w, const double *A, cudaStream_t s)
{
  if (w.n_plus > 0 && w.n_minus > 0) {
    const int n = w.n;
    k_colnorm<<<(n + 7) / 8 < 1184 ? (n + 7) / 8 : 1184, 256, 0, s>>>(w.st, A, n, w.cn);
    dim3 g((w.n_plus + GT - 1) / GT, (w.n_minus + GT - 1) / GT);
    k_gram<<<g, 128, 2 * kGramOperand, s>>>(w.st, A, w.plus, w.minus, w.n_plus, w.n_minus, n, w.gram);
    const long long np = (long long)w.n_plus * w.n_minus;
    k_hyp_gram<<<(unsigned)((np + 255) / 256), 256, 0, s>>>(w.st, A, w.plus, w.minus, w.n_plus, w.n_minus, n, w.gram,
                                                           w.cn, w.Wm);
  }
  return cudaGetLastError();
}

cudaError_t prepare_gram()
{
  return cudaFuncSetAttribute(k_gram, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(2 * kGramOperand));
}

}  // namespace jk
