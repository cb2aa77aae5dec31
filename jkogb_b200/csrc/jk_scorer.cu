// jk_scorer.cu -- the learned ranking of the scanned hyperbolic pairs (no counterpart in
// the reference, which ranks by the exact weights of DMAGF2H, src/D/dstep.F90:41-72).
//
// A hyperbolic pair whose 2x2 HSVD changes the columns needs the O(N) column scan of
// ABODNDF2 (src/D/dtransf.F90:246-348) for its weight; that scan dominates a step.  A
// scored step ranks those pairs instead by
//   w_gram = the same off-norm reduction written through the Gram matrix of the columns
//            with their diagonal removed (one FP64 matrix product per step, k_gram), and
//   w      = w_gram * 2^(clamp(y, -1, 1) / 8), y the network's learned correction
//            (no network: y = 0).
// The "no transformation" tests (NaN), the weights that need no scan, the selection, the
// 2x2 HSVDs, the rotations and the end-of-loop test stay exact.  When the off-norm has
// not reached a new minimum for `stall_k` steps the next step ranks by the exact weights,
// and only an exact step ends the loop.
//
// Network: 8 features -> 64 (ReLU) -> 64 (ReLU) -> 1, BF16 weights and inputs, FP32
// biases and accumulation, on the tensor cores (mma.sync m16n8k16, 16 pairs per warp
// and tile); the first layer's activations enter the second layer rounded to BF16.
// Features of the pair (p, q) (all log2 / 64 of magnitudes, zero counting as 2^-1074):
//   x0 |w_gram|, x1 sign(w_gram), x2 sum_{i != p,q} A(i,p)^2, x3 sum_{i != p,q} A(i,q)^2,
//   x4 |sum_{i != p,q} A(i,p) A(i,q)|, x5 |d0| (the two leading terms), x6 |Z12| + |Z21|
//   (the size of the hyperbolic transformation), x7 min(S / (10 N), 4).
// Training target: clamp(8 log2(w / w_gram), -1, 1) with w the exact weight (0 when the
// signs differ), trained by the kernels below (forward, backward into per-block partial
// gradients reduced in a fixed order, Adam) on the exact method's trajectories.
#include <cuda_bf16.h>

#include "jk_internal.h"
#include "jk_device.cuh"

namespace jk {

namespace {

constexpr int H = kMlpHidden;
constexpr int NF = kMlpFeat;
static_assert(NF == 8, "the tensor-core layer 1 reads 8 features per row (K padded to 16)");

// master parameter layout (floats): W1 [H][NF], b1 [H], W2 [H][H], b2 [H], W3 [H], b3
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + H * NF, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H, OFF_W3 = OFF_B2 + H,
              OFF_B3 = OFF_W3 + H, NPARAM = OFF_B3 + 1;
static_assert(NPARAM == mlp_params(NF), "parameter layout");
// inference layout: BF16 W1 [H][NF], W2 [H][H], W3 [H]; FP32 b1 [H], b2 [H], b3
constexpr int PW_W1 = 0, PW_W2 = H * NF, PW_W3 = PW_W2 + H * H;

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float bf16_load(unsigned short u) { return __bfloat162float(__ushort_as_bfloat16(u)); }
__device__ __forceinline__ unsigned pack_bf16(float lo, float hi)
{
  return (unsigned)__bfloat16_as_ushort(__float2bfloat16_rn(lo)) | ((unsigned)__bfloat16_as_ushort(__float2bfloat16_rn(hi)) << 16);
}

__device__ __forceinline__ float lg64(double x)
{
  const double a = fabs(x);
  return (float)(((a > 0.0) ? log2(a) : -1074.0) * (1.0 / 64.0));
}

// ---------------------------------------------------------------------------
// the network
// ---------------------------------------------------------------------------
// one block's copy of the inference parameters (shared memory)
struct TNet {
  unsigned short w1[H * NF], w2[H * H];
  float w3[H], b1[H], b2[H], b3;
};

__device__ void load_tnet(TNet &s, const unsigned short *w, const float *b)
{
  for (int k = threadIdx.x; k < H * NF; k += blockDim.x) s.w1[k] = w[PW_W1 + k];
  for (int k = threadIdx.x; k < H * H; k += blockDim.x) s.w2[k] = w[PW_W2 + k];
  for (int k = threadIdx.x; k < H; k += blockDim.x) {
    s.w3[k] = bf16_load(w[PW_W3 + k]);
    s.b1[k] = b[k];
    s.b2[k] = b[H + k];
  }
  if (threadIdx.x == 0) s.b3 = b[2 * H];
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const unsigned (&a)[4], unsigned b0, unsigned b1)
{
  asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
               "{%0, %1, %2, %3};\n"
               : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// The network on 16 feature rows xs[16][NF] (shared memory) by one warp on the tensor
// cores; y[16] (shared memory) receives the outputs.  m16n8k16 fragments: lane = 4 g + t;
// A rows g, g + 8 and columns 2t, 2t + 1 (+ 8); B column g, rows 2t, 2t + 1 (+ 8);
// C rows g, g + 8, columns 2t, 2t + 1.  Layer 1's C fragments are layer 2's A fragments.
__device__ __forceinline__ void mlp16(const TNet &s, const float (*xs)[NF], float *y)
{
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  unsigned a1[4];
  a1[0] = pack_bf16(xs[g][2 * t], xs[g][2 * t + 1]);
  a1[1] = pack_bf16(xs[g + 8][2 * t], xs[g + 8][2 * t + 1]);
  a1[2] = 0u;  // columns 8 .. 15: padding
  a1[3] = 0u;
  float h1[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int c = 8 * j + 2 * t;
    h1[j][0] = h1[j][2] = s.b1[c];
    h1[j][1] = h1[j][3] = s.b1[c + 1];
    const unsigned b0 = *(const unsigned *)&s.w1[(8 * j + g) * NF + 2 * t];
    mma_bf16(h1[j], a1, b0, 0u);
  }
  float h2[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int c = 8 * j + 2 * t;
    h2[j][0] = h2[j][2] = s.b2[c];
    h2[j][1] = h2[j][3] = s.b2[c + 1];
  }
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
    unsigned a2[4];
    a2[0] = pack_bf16(fmaxf(h1[2 * kt][0], 0.0f), fmaxf(h1[2 * kt][1], 0.0f));
    a2[1] = pack_bf16(fmaxf(h1[2 * kt][2], 0.0f), fmaxf(h1[2 * kt][3], 0.0f));
    a2[2] = pack_bf16(fmaxf(h1[2 * kt + 1][0], 0.0f), fmaxf(h1[2 * kt + 1][1], 0.0f));
    a2[3] = pack_bf16(fmaxf(h1[2 * kt + 1][2], 0.0f), fmaxf(h1[2 * kt + 1][3], 0.0f));
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const unsigned short *row = &s.w2[(8 * j + g) * H + 16 * kt + 2 * t];
      mma_bf16(h2[j], a2, *(const unsigned *)row, *(const unsigned *)(row + 8));
    }
  }
  float y0 = 0.0f, y1 = 0.0f;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int c = 8 * j + 2 * t;
    y0 = fmaf(s.w3[c], fmaxf(h2[j][0], 0.0f), y0);
    y0 = fmaf(s.w3[c + 1], fmaxf(h2[j][1], 0.0f), y0);
    y1 = fmaf(s.w3[c], fmaxf(h2[j][2], 0.0f), y1);
    y1 = fmaf(s.w3[c + 1], fmaxf(h2[j][3], 0.0f), y1);
  }
  y0 += __shfl_xor_sync(0xFFFFFFFFu, y0, 1);
  y0 += __shfl_xor_sync(0xFFFFFFFFu, y0, 2);
  y1 += __shfl_xor_sync(0xFFFFFFFFu, y1, 1);
  y1 += __shfl_xor_sync(0xFFFFFFFFu, y1, 2);
  if (t == 0) {
    y[g] = y0 + s.b3;
    y[g + 8] = y1 + s.b3;
  }
}

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

// column off-diagonal norms cn[j] = sum_{i != j} |A(i,j)|^2 (one warp per column; C = 2:
// complex A, each column read as 2 n interleaved reals)
template <int C>
__global__ void __launch_bounds__(256)
k_colnorm(const State *st, const double *__restrict__ A, int n, double *__restrict__ cn)
{
  if (st->stop || !st->learned_step) return;
  const int lane = threadIdx.x & 31;
  for (int j = blockIdx.x * 8 + (threadIdx.x >> 5); j < n; j += gridDim.x * 8) {
    const double *c = A + (long long)j * C * n;
    double s = 0.0;
    for (int i = lane; i < C * n; i += 32)
      if (i / C != j) s = fma(c[i], c[i], s);
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

// C = 1: real A; C = 2: complex A, read as 2 n interleaved reals per column, so that the
// real product of two columns is Re(x^H y); IM: the B operand's (re, im) pairs are read as
// (im, -re), which makes the product Im(x^H y)
template <int C, bool IM>
__device__ __forceinline__ void gram_tile(const double *__restrict__ A, const int *__restrict__ plus,
                                          const int *__restrict__ minus, int n_plus, int n_minus, int n,
                                          double *__restrict__ G)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double (*xs)[GT][GKP] = (double (*)[GT][GKP])smem_raw;            // [2][GT][GKP]
  double (*ys)[GT][GKP] = (double (*)[GT][GKP])(smem_raw + kGramOperand);
  __shared__ int cx[GT], cy[GT];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int a0 = blockIdx.x * GT, b0 = blockIdx.y * GT;
  const int nd = C * n;  // reals per column
  if (tid < GT) {
    cx[tid] = (a0 + tid < n_plus) ? plus[a0 + tid] : -1;
    cy[tid] = (b0 + tid < n_minus) ? minus[b0 + tid] : -1;
  }
  __syncthreads();
  const int nk = (nd + GK - 1) / GK;
  // staging: 2 operands x 64 columns x 16 pieces of 16 bytes (two reals each) = 2048
  // copies, 16 per thread; a piece that is not 16-byte aligned in A or runs past the
  // column's end is loaded by plain loads (zeros past the end)
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
        const long long e = (long long)g * nd + r;
        if (g >= 0 && r + 1 < nd && !(e & 1)) cp_async16g(dst, A + e, true);  // 16-byte aligned piece
        else {
          dst[0] = (g >= 0 && r < nd) ? A[e] : 0.0;
          dst[1] = (g >= 0 && r + 1 < nd) ? A[e + 1] : 0.0;
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
      const int kr = kk + fk;             // this lane's real index in the chunk
      const int row = (k0 + kr) / C;      // the matrix row it belongs to
      double fa[4], fb[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        fa[i] = (row == gxa[i]) ? 0.0 : xs[buf][wm + 8 * i + fr][kr];
        double b;
        if constexpr (IM) b = (kr & 1) ? -ys[buf][wn + 8 * i + fr][kr - 1] : ys[buf][wn + 8 * i + fr][kr + 1];
        else b = ys[buf][wn + 8 * i + fr][kr];
        fb[i] = (row == gyb[i]) ? 0.0 : b;
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

// the Gram products of a scored step: G[a][b] (real A); Re and Im of x_a^H y_b (complex A,
// blockIdx.z 0 and 1, the imaginary parts n_plus n_minus entries after the real ones)
template <int C>
__global__ void __launch_bounds__(128)
k_gram(const State *st, const double *__restrict__ A, const int *__restrict__ plus, const int *__restrict__ minus,
       int n_plus, int n_minus, int n, double *__restrict__ G)
{
  if (st->stop || !st->learned_step) return;
  if (C == 2 && blockIdx.z) gram_tile<C, true>(A, plus, minus, n_plus, n_minus, n, G + (long long)n_plus * n_minus);
  else gram_tile<C, false>(A, plus, minus, n_plus, n_minus, n, G);
}



// ---------------------------------------------------------------------------
// a pair of a scored step: the exact 2x2 part of DMAGF2H and, for a pair that needs the
// column scan, the Gram form of its weight and its features (rounded to BF16)
// ---------------------------------------------------------------------------
struct GPair {
  double w;     // the weight (exact, or w_gram for a scanned pair)
  int scan;     // the pair needs the column scan
  float x[NF];  // features of a scanned pair
};

__device__ __forceinline__ GPair gram_pair(const double *__restrict__ A, int n, int a, int b, long long gidx, long long,
                                           const double *__restrict__ G, const double *__restrict__ cn, int step)
{
  GPair r;
  r.w = nan_w();
  r.scan = 0;
  const bool a_is_p = a < b;
  const int p = a_is_p ? a : b, q = a_is_p ? b : a;
  const double app = A[(long long)p * n + p], aqp = A[(long long)p * n + q], apq = A[(long long)q * n + p],
               aqq = A[(long long)q * n + q];
  if (!may_transform(app, aqp, apq, aqq)) return r;
  double A2[4] = { app, aqp, apq, aqq }, U2[4], Z2[4];
  int info = 0;
  const int jp = a_is_p ? 1 : -1;
  dhsvd2(A2, jp, -jp, U2, Z2, JK_TH1FIX, info);
  if (info < 0) return r;
  if (!(info & 1)) { r.w = 0.0; return r; }
  if (!(info & 4)) { r.w = dasum2(aqp, apq); return r; }
  const double a1 = (info & 8) ? A2[M21] : 0.0, a2 = (info & 8) ? A2[M12] : 0.0;
  double d = 0.0;
  d = fma(__dsub_rn(aqp, a1), __dadd_rn(aqp, a1), d);
  d = fma(__dsub_rn(apq, a2), __dadd_rn(apq, a2), d);
  const double z11 = Z2[M11], z21 = Z2[M21], z12 = Z2[M12], z22 = Z2[M22];
  const double nx = cn[p] - aqp * aqp, ny = cn[q] - apq * apq;
  const double g = G[gidx];
  // 1 - z11^2 - z12^2 and 1 - z21^2 - z22^2 without cancellation at z11, z22 near +-1
  const double c1 = (1.0 - z11) * (1.0 + z11) - z12 * z12;
  const double c2 = (1.0 - z22) * (1.0 + z22) - z21 * z21;
  const double c3 = z11 * z21 + z12 * z22;
  r.w = d + (nx * c1 + ny * c2 - 2.0 * c3 * g);
  r.scan = 1;
  r.x[0] = bf16_round(lg64(r.w));
  r.x[1] = (r.w < 0.0) ? -1.0f : 1.0f;
  r.x[2] = bf16_round(lg64(nx));
  r.x[3] = bf16_round(lg64(ny));
  r.x[4] = bf16_round(lg64(g));
  r.x[5] = bf16_round(lg64(d));
  r.x[6] = bf16_round(lg64(fabs(z12) + fabs(z21)));
  r.x[7] = bf16_round(fminf((float)step / (10.0f * (float)n), 4.0f));
  return r;
}

// the complex pair (ZMAGF2H, src/Z/zstep.F90:43-74): with x, y the columns p, q without
// rows p, q and g = x^H y (the Gram product of the "+" and "-" columns, conjugated when the
// "-" column comes first), the scan's sum is d + nx (1 - |Z11|^2 - |Z12|^2) +
// ny (1 - |Z21|^2 - |Z22|^2) - 2 Re((conj(Z11) Z21 + conj(Z12) Z22) g)
__device__ __forceinline__ GPair gram_pair(const double2 *__restrict__ A, int n, int a, int b, long long gidx,
                                           long long npm, const double *__restrict__ G, const double *__restrict__ cn,
                                           int step)
{
  GPair r;
  r.w = nan_w();
  r.scan = 0;
  const bool a_is_p = a < b;
  const int p = a_is_p ? a : b, q = a_is_p ? b : a;
  const double2 app = A[(long long)p * n + p], aqp = A[(long long)p * n + q], apq = A[(long long)q * n + p],
                aqq = A[(long long)q * n + q];
  if (!may_transform(app, aqp, apq, aqq)) return r;
  double2 A2[4] = { app, aqp, apq, aqq }, U2[4], Z2[4];
  int info = 0;
  const int jp = a_is_p ? 1 : -1;
  zhsvd2(A2, jp, -jp, U2, Z2, JK_TH1FIX, info);
  if (info < 0) return r;
  if (!(info & 1)) { r.w = 0.0; return r; }
  if (!(info & 4)) { r.w = dasum4(aqp.x, aqp.y, apq.x, apq.y); return r; }
  const double2 a1 = (info & 8) ? A2[M21] : make_double2(0.0, 0.0);
  const double2 a2 = (info & 8) ? A2[M12] : make_double2(0.0, 0.0);
  double d = 0.0;
  d = fma(__dsub_rn(aqp.x, a1.x), __dadd_rn(aqp.x, a1.x), d);
  d = fma(__dsub_rn(aqp.y, a1.y), __dadd_rn(aqp.y, a1.y), d);
  d = fma(__dsub_rn(apq.x, a2.x), __dadd_rn(apq.x, a2.x), d);
  d = fma(__dsub_rn(apq.y, a2.y), __dadd_rn(apq.y, a2.y), d);
  const double2 z11 = Z2[M11], z21 = Z2[M21], z12 = Z2[M12], z22 = Z2[M22];
  const double nx = cn[p] - (aqp.x * aqp.x + aqp.y * aqp.y), ny = cn[q] - (apq.x * apq.x + apq.y * apq.y);
  const double gr = G[gidx], gi = a_is_p ? G[npm + gidx] : -G[npm + gidx];
  const double c1 = (1.0 - z11.x) * (1.0 + z11.x) - z11.y * z11.y - (z12.x * z12.x + z12.y * z12.y);
  const double c2 = (1.0 - z22.x) * (1.0 + z22.x) - z22.y * z22.y - (z21.x * z21.x + z21.y * z21.y);
  // c3 = conj(z11) z21 + conj(z12) z22
  const double c3r = (z11.x * z21.x + z11.y * z21.y) + (z12.x * z22.x + z12.y * z22.y);
  const double c3i = (z11.x * z21.y - z11.y * z21.x) + (z12.x * z22.y - z12.y * z22.x);
  r.w = d + (nx * c1 + ny * c2 - 2.0 * (c3r * gr - c3i * gi));
  r.scan = 1;
  r.x[0] = bf16_round(lg64(r.w));
  r.x[1] = (r.w < 0.0) ? -1.0f : 1.0f;
  r.x[2] = bf16_round(lg64(nx));
  r.x[3] = bf16_round(lg64(ny));
  r.x[4] = bf16_round(lg64(hypot(gr, gi)));
  r.x[5] = bf16_round(lg64(d));
  r.x[6] = bf16_round(lg64(zabs(z12) + zabs(z21)));
  r.x[7] = bf16_round(fminf((float)step / (10.0f * (float)n), 4.0f));
  return r;
}

// the score of a scanned pair from the network's output
__device__ __forceinline__ double corrected(double w, float y) { return w * exp2((double)fminf(fmaxf(y, -1.0f), 1.0f) * 0.125); }

// the weights of the hyperbolic pairs in a scored step (one thread per pair, (+, -) order);
// with a network, every warp scores its 32 pairs as two tiles of 16 on the tensor cores
template <typename T>
__global__ void __launch_bounds__(256)
k_hyp_gram(const State *st, const T *__restrict__ A, const int *__restrict__ plus, const int *__restrict__ minus,
           int n_plus, int n_minus, int n, const double *__restrict__ G, const double *__restrict__ cn,
           double *__restrict__ Wm, ScorerDev sc)
{
  if (st->stop || !st->learned_step) return;
  __shared__ TNet net;
  __shared__ float xs[8][32][NF];
  __shared__ float ys[8][32];
  const bool with_net = (sc.nf == NF);
  if (with_net) load_tnet(net, sc.w, sc.b);
  __syncthreads();
  const long long k = blockIdx.x * 256LL + threadIdx.x;
  const bool valid = k < (long long)n_plus * n_minus;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int ia = 0, ib = 0;
  GPair r;
  r.w = nan_w();
  r.scan = 0;
  if (valid) {
    ia = (int)(k / n_minus);
    ib = (int)(k % n_minus);
    r = gram_pair(A, n, plus[ia], minus[ib], (long long)ia * n_minus + ib, (long long)n_plus * n_minus, G, cn,
                  st->steps);
  }
  if (with_net && __any_sync(0xFFFFFFFFu, r.scan)) {
#pragma unroll
    for (int f = 0; f < NF; ++f) xs[warp][lane][f] = r.scan ? r.x[f] : 0.0f;
    __syncwarp();
    mlp16(net, xs[warp], ys[warp]);
    mlp16(net, xs[warp] + 16, ys[warp] + 16);
    __syncwarp();
    if (r.scan) r.w = corrected(r.w, ys[warp][lane]);
  }
  if (!valid) return;
  double w = r.w;
  if (w < -JK_HUGE) w = nan_w();
  const int a = plus[ia], b = minus[ib];
  const int p = a < b ? a : b, q = a < b ? b : a;
  Wm[(long long)q * n + p] = w;
  Wm[(long long)p * n + q] = w;
}

// training data: the features and w_gram of every hyperbolic pair ((+, -) order); the
// pairs that need no scan get zero features and a NaN w_gram
template <typename T>
__global__ void __launch_bounds__(256)
k_gram_features(const T *__restrict__ A, const int *__restrict__ plus, const int *__restrict__ minus, int n_plus,
                int n_minus, int n, const double *__restrict__ G, const double *__restrict__ cn, int step, float *X,
                double *Wg)
{
  const long long k = blockIdx.x * 256LL + threadIdx.x;
  if (k >= (long long)n_plus * n_minus) return;
  const int ia = (int)(k / n_minus), ib = (int)(k % n_minus);
  const GPair r = gram_pair(A, n, plus[ia], minus[ib], k, (long long)n_plus * n_minus, G, cn, step);
#pragma unroll
  for (int f = 0; f < NF; ++f) X[k * NF + f] = r.scan ? r.x[f] : 0.0f;
  if (Wg) Wg[k] = r.scan ? r.w : nan_w();
}

// the off-norm sum_{i != j} A(i,j)^2 after a scored step, in a fixed summation order
// (per-block tree sums, then the last block adds the block sums in block order), and
// the choice of the next step's ranking
__device__ __forceinline__ double sq_acc(double a, double acc) { return fma(a, a, acc); }
__device__ __forceinline__ double sq_acc(double2 a, double acc) { return fma(a.y, a.y, fma(a.x, a.x, acc)); }

template <typename T>
__global__ void __launch_bounds__(256)
k_offnorm(State *st, const T *__restrict__ A, int n, double *part, int *count)
{
  if (st->stop || !st->learned) return;
  __shared__ double red[256];
  __shared__ int last;
  const long long nn = (long long)n * n;
  double acc = 0.0;
  for (long long k = blockIdx.x * 256LL + threadIdx.x; k < nn; k += (long long)gridDim.x * 256) {
    const int i = (int)(k % n), j = (int)(k / n);
    if (i != j) acc = sq_acc(A[k], acc);
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
    // no effective pivot among the scored choices: the end-of-loop test is left to an
    // exact step
    st->retry = 1;
    st->learned_step = 0;
    st->stall = 0;
    st->exact_steps += 1;
    return;
  }
  if (off > 16.0 * st->best_off) {
    // the scored choices let the off-norm grow: the rest of the solve ranks exactly
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
// training
// ---------------------------------------------------------------------------
// the network's output on `count` feature rows with the inference parameters (tensor cores)
__global__ void __launch_bounds__(256)
k_mlp_forward(const float *__restrict__ X, const unsigned short *__restrict__ w, const float *__restrict__ b, int count, float *Y)
{
  __shared__ TNet net;
  __shared__ float xs[8][32][NF];
  __shared__ float ys[8][32];
  load_tnet(net, w, b);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long s = blockIdx.x * 256LL + threadIdx.x;
#pragma unroll
  for (int f = 0; f < NF; ++f) xs[warp][lane][f] = (s < count) ? bf16_round(X[s * NF + f]) : 0.0f;
  __syncwarp();
  mlp16(net, xs[warp], ys[warp]);
  mlp16(net, xs[warp] + 16, ys[warp] + 16);
  __syncwarp();
  if (s < count) Y[s] = ys[warp][lane];
}

// the network's weights in FP32 from the master parameters, rounded to BF16 as inference
// uses them (shared memory)
struct SNet {
  float w1[H * NF], b1[H], w2[H * H], b2[H], w3[H], b3;
};

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

constexpr int GB = 128;  // samples per block of the gradient kernel

// loss = mean (y - t)^2 over `count` samples; this block's partial gradient (and loss)
// of its GB samples into part[blockIdx.x][NPARAM + 1].  The forward pass is the
// inference arithmetic in scalar form (BF16 inputs and weights, layer 1's activations
// rounded to BF16, FP32 sums); the rounding of the activations passes the gradient
// through unchanged.
__global__ void __launch_bounds__(GB)
k_mlp_grad(const float *__restrict__ X, const float *__restrict__ T, const float *__restrict__ P, int count, float *part)
{
  __shared__ SNet net;
  extern __shared__ float dyn[];
  float *h1 = dyn;               // [GB][H] activations (BF16-rounded), later their gradients
  float *h2 = h1 + GB * H;       // [GB][H] activations, later their gradients
  float *xs = h2 + GB * H;       // [GB][NF]
  float *dy = xs + GB * NF;      // [GB]
  load_net_master(net, P);
  const int tid = threadIdx.x, s = blockIdx.x * GB + tid;
  const bool valid = s < count;
  const float inv = 1.0f / (float)count;
  float x[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) { x[f] = valid ? bf16_round(X[(long long)s * NF + f]) : 0.0f; xs[tid * NF + f] = x[f]; }
  __syncthreads();
  float y = net.b3;
  for (int j = 0; j < H; ++j) {
    float a = net.b1[j];
#pragma unroll
    for (int f = 0; f < NF; ++f) a = fmaf(net.w1[j * NF + f], x[f], a);
    h1[tid * H + j] = bf16_round(fmaxf(a, 0.0f));
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
  // dW3, db3
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
  if (k < H * NF) w[PW_W1 + k] = __bfloat16_as_ushort(__float2bfloat16_rn(P[OFF_W1 + k]));
  if (k < H * H) w[PW_W2 + k] = __bfloat16_as_ushort(__float2bfloat16_rn(P[OFF_W2 + k]));
  if (k < H) {
    w[PW_W3 + k] = __bfloat16_as_ushort(__float2bfloat16_rn(P[OFF_W3 + k]));
    b[k] = P[OFF_B1 + k];
    b[H + k] = P[OFF_B2 + k];
  }
  if (k == 0) b[2 * H] = P[OFF_B3];
}

}  // namespace

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
template <typename T>
static cudaError_t learned_weights_t(Workspace &w, const T *A, cudaStream_t s)
{
  constexpr int C = sizeof(T) / sizeof(double);
  if (w.n_plus > 0 && w.n_minus > 0) {
    const int n = w.n;
    k_colnorm<C><<<(n + 7) / 8 < 1184 ? (n + 7) / 8 : 1184, 256, 0, s>>>(w.st, (const double *)A, n, w.cn);
    dim3 g((w.n_plus + GT - 1) / GT, (w.n_minus + GT - 1) / GT, C);
    k_gram<C><<<g, 128, 2 * kGramOperand, s>>>(w.st, (const double *)A, w.plus, w.minus, w.n_plus, w.n_minus, n, w.gram);
    const long long np = (long long)w.n_plus * w.n_minus;
    k_hyp_gram<T><<<(unsigned)((np + 255) / 256), 256, 0, s>>>(w.st, A, w.plus, w.minus, w.n_plus, w.n_minus, n,
                                                              w.gram, w.cn, w.Wm, w.sc);
  }
  return cudaGetLastError();
}

cudaError_t launch_learned_weights(Workspace &w, const void *A, cudaStream_t s)
{
  return w.cplx ? learned_weights_t(w, (const double2 *)A, s) : learned_weights_t(w, (const double *)A, s);
}

cudaError_t prepare_gram()
{
  const int sm = (int)(2 * kGramOperand);
  cudaError_t e = cudaFuncSetAttribute(k_gram<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_gram<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  return e;
}

cudaError_t launch_offnorm(Workspace &w, const void *A, cudaStream_t s)
{
  if (w.cplx) k_offnorm<double2><<<kOffBlocks, 256, 0, s>>>(w.st, (const double2 *)A, w.n, w.offpart, w.offcount);
  else k_offnorm<double><<<kOffBlocks, 256, 0, s>>>(w.st, (const double *)A, w.n, w.offpart, w.offcount);
  return cudaGetLastError();
}

template <typename T>
static cudaError_t features_t(int n, const T *A, const int *plus, const int *minus, int n_plus, int n_minus, int step,
                              const State *st, double *G, double *cn, float *X, double *Wg, cudaStream_t s)
{
  constexpr int C = sizeof(T) / sizeof(double);
  const long long cnt = (long long)n_plus * n_minus;
  k_colnorm<C><<<(n + 7) / 8 < 1184 ? (n + 7) / 8 : 1184, 256, 0, s>>>(st, (const double *)A, n, cn);
  dim3 g((n_plus + GT - 1) / GT, (n_minus + GT - 1) / GT, C);
  k_gram<C><<<g, 128, 2 * kGramOperand, s>>>(st, (const double *)A, plus, minus, n_plus, n_minus, n, G);
  k_gram_features<T><<<(unsigned)((cnt + 255) / 256), 256, 0, s>>>(A, plus, minus, n_plus, n_minus, n, G, cn, step, X,
                                                                    Wg);
  return cudaGetLastError();
}

cudaError_t mlp_features(int cplx, int n, const void *A, const int *plus, const int *minus, int n_plus, int n_minus,
                         int step, const State *st, double *G, double *cn, float *X, double *Wg, cudaStream_t s)
{
  const long long cnt = (long long)n_plus * n_minus;
  if (cnt <= 0) return cudaSuccess;
  cudaError_t e = prepare_gram();
  if (e != cudaSuccess) return e;
  return cplx ? features_t(n, (const double2 *)A, plus, minus, n_plus, n_minus, step, st, G, cn, X, Wg, s)
              : features_t(n, (const double *)A, plus, minus, n_plus, n_minus, step, st, G, cn, X, Wg, s);
}

cudaError_t mlp_forward(int nf, int count, const float *X, const unsigned short *w, const float *b, float *Y, cudaStream_t s)
{
  if (nf != NF) return cudaErrorInvalidValue;
  if (count > 0) k_mlp_forward<<<(count + 255) / 256, 256, 0, s>>>(X, w, b, count, Y);
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
