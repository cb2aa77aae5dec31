// jk_kernels.cu -- the per-step CUDA kernels of the J-Kogbetliantz HSVD (real and
// complex), B200 (sm_100a).  One step of DSTEP_EXEC / ZSTEP_EXEC
// (src/D/dstep.F90:376-443, src/Z/zstep.F90:379-447) is seven launches:
//
//   k_weights_trig  pair weights of the trigonometric pairs      (DMAGF2T / ZMAGF2T)
//   k_weights_hyp   pair weights of the hyperbolic pairs         (DMAGF2H / ZMAGF2H)
//                   = batched 2x2 HSVD + the tiled off-norm scan (ABODNDF2 / ABODNZF2)
//   k_colsort       every vertex's partners ranked by the records' sort order (AW_CMP)
//   k_select        one block: the end-of-step test of the previous step
//                   (SL := MIN(SL, NL)); the greedy non-colliding selection of the
//                   sorted records (AW_SRT* + AW_NCP1/2) as the greedy matching, in
//                   rounds of mutual best proposals; the ranking of the matched pairs
//                   and the first N_2 of them
//   k_pivots        the 2x2 HSVD of every selected pivot (DHSVD2 / ZHSVD2), INFO, NL
//   k_rotate        fused transformations: every block loads a column pair of A,
//                   applies all row rotations (BA), then its column rotation (AB)
//                   and the diagonal write-back, and rotates the columns of U and Z
//
// Matrices are column-major with leading dimension n; complex entries are double2.
#include <cooperative_groups.h>

#include <cstdlib>
#include <cstring>
#include <mutex>

#include "jk_internal.h"
#include "jk_device.cuh"

namespace cg = cooperative_groups;

namespace jk {

// ---------------------------------------------------------------------------
// initialisation and finalisation
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_identity2(T *U, T *Z, int n)
{
  const long long nn = (long long)n * n;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nn; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % n), j = (int)(k / n);
    const T v = (i == j) ? Tr<T>::one() : Tr<T>::zero();
    U[k] = v;
    Z[k] = v;
  }
}

// the loop state at the start of a solve (S = steps0; 0 for a new solve); the trace
// capacities are kept, the learned-ranking settings are the caller's
__global__ void k_state_init(State *st, int learned, int stall_k, int steps0)
{
  const int cap_s = st->trace_cap_steps, on = st->trace_on;
  const long long cap_p = st->trace_cap_piv;
  State z = {};
  z.trace_on = on;
  z.trace_cap_steps = cap_s;
  z.trace_cap_piv = cap_p;
  z.tw = -0.0;
  z.steps = steps0;
  z.learned = learned;
  z.learned_step = learned;
  z.stall_k = stall_k;
  z.best_off = __longlong_as_double(0x7FF0000000000000LL);  // +inf
  *st = z;
}

// a new step limit; a loop waiting at the old one goes on
__global__ void k_set_limit(State *st, long long limit)
{
  if (st->stop == 2) st->stop = 0;
  st->limit = limit;
}

// A(i,i) := SIGMA(i): the loop's matrix back from what the end of the loop made of it
template <typename T>
__global__ void k_unsigma(T *A, const double *sigma, int n)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    T v = Tr<T>::zero();
    *(double *)&v = sigma[i];
    A[(long long)i * n + i] = v;
  }
}

// SIGMA(S) = A(S,S); A(S,S) = 0   (src/D/dstep.F90:594-602, src/Z/zstep.F90:605-613)
template <typename T>
__global__ void k_sigma(T *A, double *sigma, int n)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const long long k = (long long)i * n + i;
    sigma[i] = Tr<T>::re(A[k]);
    A[k] = Tr<T>::zero();
  }
}

// Z := J Z^T J (JZTJ, src/D/dstep.F90:447-468) or J Z^H J (JZHJ, src/Z/zstep.F90:451-478),
// in place, one 32x32 tile pair per block
template <typename T>
__global__ void k_jztj(T *Z, const int *J, int n)
{
  __shared__ T a[32][33], b[32][33];
  const int nt = (n + 31) / 32;
  // block -> (ti, tj), ti <= tj
  int t = blockIdx.x, ti = 0;
  while (t >= nt - ti) { t -= nt - ti; ++ti; }
  const int tj = ti + t;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int r = ty; r < 32; r += blockDim.y) {
    const int i1 = ti * 32 + tx, j1 = tj * 32 + r;  // tile (ti, tj): rows ti, cols tj
    const int i2 = tj * 32 + tx, j2 = ti * 32 + r;  // tile (tj, ti)
    if (i1 < n && j1 < n) a[r][tx] = Z[(long long)j1 * n + i1];
    if (i2 < n && j2 < n) b[r][tx] = Z[(long long)j2 * n + i2];
  }
  __syncthreads();
  for (int r = ty; r < 32; r += blockDim.y) {
    // new Z(i, j) = J_i conj(Z(j, i)) J_j
    const int i1 = ti * 32 + tx, j1 = tj * 32 + r;
    if (i1 < n && j1 < n && (ti != tj || i1 <= j1)) {
      T v = Tr<T>::conj_(b[tx][r]);            // old Z(j1, i1)
      if (i1 != j1 && J[i1] != J[j1]) v = Tr<T>::neg_(v);
      if (ti == tj && i1 == j1) v = Tr<T>::conj_(a[r][tx]);
      Z[(long long)j1 * n + i1] = v;
    }
    const int i2 = tj * 32 + tx, j2 = ti * 32 + r;
    if (ti != tj && i2 < n && j2 < n) {
      T v = Tr<T>::conj_(a[tx][r]);            // old Z(j2, i2)
      if (J[i2] != J[j2]) v = Tr<T>::neg_(v);
      Z[(long long)j2 * n + i2] = v;
    }
  }
  if (ti == tj) {
    // the lower half of a diagonal tile
    __syncthreads();
    for (int r = ty; r < 32; r += blockDim.y) {
      const int i1 = ti * 32 + tx, j1 = tj * 32 + r;
      if (i1 < n && j1 < n && i1 > j1) {
        T v = Tr<T>::conj_(a[tx][r]);
        if (J[i1] != J[j1]) v = Tr<T>::neg_(v);
        Z[(long long)j1 * n + i1] = v;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// weights of the trigonometric pairs: DMAGF2T (src/D/dstep.F90:12-37),
// ZMAGF2T (src/Z/zstep.F90:12-39); one thread per (p, q), both halves of Wm written
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_weights_trig(const State *st, const T *__restrict__ A, const int *__restrict__ J, double *__restrict__ Wm, int n)
{
  if (st->stop) return;
  const int p = blockIdx.x * 32 + threadIdx.x, q = blockIdx.y * 8 + threadIdx.y;
  if (p >= n || q >= n || p >= q) return;
  const int s = J[p] + J[q];
  if (s != 2 && s != -2) return;  // hyperbolic pairs are the other kernel's
  const T app = A[(long long)p * n + p], aqp = A[(long long)p * n + q], apq = A[(long long)q * n + p], aqq = A[(long long)q * n + q];
  const bool nz = may_transform(app, aqp, apq, aqq);
  double w;
  if (s == -2) w = (nz || (Tr<T>::re(aqq) < Tr<T>::re(app))) ? Tr<T>::magt(aqp, apq) : nan_w();
  else w = (nz || (Tr<T>::re(app) < Tr<T>::re(aqq))) ? Tr<T>::magt(aqp, apq) : nan_w();
  Wm[(long long)q * n + p] = w;
  Wm[(long long)p * n + q] = w;
}

// ---------------------------------------------------------------------------
// weights of the hyperbolic pairs: DMAGF2H (src/D/dstep.F90:41-72) with ABODNDF2
// (src/D/dtransf.F90:246-348), ZMAGF2H (src/Z/zstep.F90:43-74) with ABODNZF2
// (src/Z/ztransf.F90:452-637).  A block owns HP "+" columns x HM "-" columns; each
// thread owns one pair and keeps the reference's sequential row order in its own
// fma chain, while the column data are staged through shared memory in row chunks
// and reused by the whole tile.  The -inf of a weight becomes NaN (src/D/dstep.F90:212-214).
// ---------------------------------------------------------------------------
#define HR 64

__device__ __forceinline__ void scan_rows_real(const double *xs, const double *ys, int rows, int i0, int p, int q, const Rot &t, double &d)
{
  if (t.c1 && t.c2) {
#pragma unroll 4
    for (int r = 0; r < rows; ++r) {
      const double x = xs[r], y = ys[r];
      const double xx = __dmul_rn(fma(y, t.r1, x), t.m1);
      const double yy = __dmul_rn(fma(x, t.r2, y), t.m2);
      const int i = i0 + r;
      if (i != p && i != q) {
        d = fma(__dsub_rn(x, xx), __dadd_rn(x, xx), d);
        d = fma(__dsub_rn(y, yy), __dadd_rn(y, yy), d);
      }
    }
  }
  else {
    for (int r = 0; r < rows; ++r) {
      double x = xs[r], y = ys[r];
      const double x0 = x, y0 = y;
      rot_apply(t, x, y);
      const int i = i0 + r;
      if (i != p && i != q) {
        d = fma(__dsub_rn(x0, x), __dadd_rn(x0, x), d);
        d = fma(__dsub_rn(y0, y), __dadd_rn(y0, y), d);
      }
    }
  }
}

__device__ __forceinline__ void scan_rows_cplx(const double2 *xs, const double2 *ys, int rows, int i0, int p, int q, const ZRot &t, double &d)
{
  for (int r = 0; r < rows; ++r) {
    double2 x = xs[r], y = ys[r];
    const double2 x0 = x, y0 = y;
    zrot_apply_ab(t, x, y);
    const int i = i0 + r;
    if (i != p && i != q) {
      const double axi = zabs(x0), axx = zabs(x), ayi = zabs(y0), ayy = zabs(y);
      d = fma(__dsub_rn(axi, axx), __dadd_rn(axi, axx), d);
      d = fma(__dsub_rn(ayi, ayy), __dadd_rn(ayi, ayy), d);
    }
  }
}

// ---------------------------------------------------------------------------
// the real hyperbolic weights, pipelined: a block owns 16 "+" columns x 32 "-"
// columns; each thread owns two pairs sharing its "+" column (two independent fma
// chains); row chunks of the 48 columns stream into a double buffer in shared
// memory with cp.async while the previous chunk is consumed.
// ---------------------------------------------------------------------------

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// the 2x2 part of DMAGF2H for one pair of A (global, leading dimension n)
__device__ __forceinline__ bool hyp_pair_setup(const double *__restrict__ A, int n, int a, int b, int &p, int &q, bool &a_is_p,
                                               double &w, double &d, Rot &t)
{
  a_is_p = (a < b);
  p = a_is_p ? a : b;
  q = a_is_p ? b : a;
  return hyp_setup(A[(long long)p * n + p], A[(long long)p * n + q], A[(long long)q * n + p], A[(long long)q * n + q],
                   a_is_p ? 1 : -1, w, d, t);
}

// The real hyperbolic weights, pipelined (k_hyp_pm below): sign-class tiles of 32 "+"
// by 32 "-" vertices, 64 rows per chunk staged with cp.async, the sequential ABODNDF2
// fma chains of four pairs per thread.
#define TW 32
#define SCAN_ROWS 64
#define SCAN_RS (SCAN_ROWS + 2)

// rows of a chunk unrolled together in the scan (a tuning knob; 2 unless set at build time)
#ifndef JK_SCAN_UNROLL
#define JK_SCAN_UNROLL 2
#endif
constexpr int kScanUnroll = JK_SCAN_UNROLL;

// Two rows (r, r + 1 of the chunk) of K pairs' ABODNDF2 chains.  TEST: some pair of the
// warp has its row p or q among them, so every pair skips its own p and q; inactive slots
// accumulate garbage that is never stored (a predicated pair of fmas instead of a select
// of their result).
template <int K, bool TEST, bool FULL>
__device__ __forceinline__ void scan_rows2(const double2 *xv, const double2 *yv, int r, int rows, const int *pl,
                                           const int *ql, const double *r1, const double *r2, const double *m1,
                                           const double *m2, double *d)
{
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    if (!FULL && h == 1 && r + 1 >= rows) break;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const double x = h ? xv[k].y : xv[k].x, y = h ? yv[k].y : yv[k].x;
      const double xx = __dmul_rn(fma(y, r1[k], x), m1[k]);
      const double yy = __dmul_rn(fma(x, r2[k], y), m2[k]);
      const double s1 = __dsub_rn(x, xx), a1 = __dadd_rn(x, xx), s2 = __dsub_rn(y, yy), a2 = __dadd_rn(y, yy);
      if (!TEST || ((r + h) != pl[k] && (r + h) != ql[k])) {
        d[k] = fma(s1, a1, d[k]);
        d[k] = fma(s2, a2, d[k]);
      }
    }
  }
}

// rows of a chunk that share one decision whether to run the skip test (a tuning knob)
#ifndef JK_SCAN_SUB
#define JK_SCAN_SUB 32
#endif
constexpr int kScanSub = JK_SCAN_SUB;
static_assert(SCAN_ROWS % kScanSub == 0 && kScanSub % 2 == 0, "sub-blocks tile the chunk in row pairs");

// rows r0 .. r0 + kScanSub - 1 of a full chunk
template <int K, int SHARED, bool TEST>
__device__ __forceinline__ void scan_sub(const double *const *xs, const double *const *ys, const double *sh, int r0,
                                         const int *pl, const int *ql, const double *r1, const double *r2,
                                         const double *m1, const double *m2, double *d)
{
#pragma unroll kScanUnroll
  for (int r = r0; r < r0 + kScanSub; r += 2) {
    double2 xv[K], yv[K];
    double2 sv = make_double2(0.0, 0.0);
    if (SHARED) sv = *(const double2 *)(sh + r);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      xv[k] = (SHARED == 2) ? sv : *(const double2 *)(xs[k] + r);
      yv[k] = (SHARED == 1) ? sv : *(const double2 *)(ys[k] + r);
    }
    scan_rows2<K, TEST, true>(xv, yv, r, SCAN_ROWS, pl, ql, r1, r2, m1, m2, d);
  }
}

// One row chunk of K pairs per thread (slots t, t + 256, ...).  SHARED 0: pair k scans
// columns xs[k] (its p) and ys[k] (its q); SHARED 1: every pair's q column is `sh` (one
// load serves all K); SHARED 2: every pair's p column is `sh`.  `touch` (warp-uniform)
// marks the chunk's rows that are some pair's p or q: only the sub-blocks of kScanSub
// rows that hold one run the skip test.  FULL: the chunk has all SCAN_ROWS rows; the
// last, shorter chunk always runs the test.
template <int K, int SHARED, bool FULL>
__device__ __forceinline__ void scan_chunk(const double *const *xs, const double *const *ys, const double *sh,
                                           const int *pl, const int *ql, const double *r1, const double *r2,
                                           const double *m1, const double *m2, double *d, int rows,
                                           unsigned long long touch)
{
  if constexpr (FULL) {
#pragma unroll 1
    for (int r0 = 0; r0 < SCAN_ROWS; r0 += kScanSub) {
      if ((touch >> r0) & ((2ull << (kScanSub - 1)) - 1ull)) scan_sub<K, SHARED, true>(xs, ys, sh, r0, pl, ql, r1, r2, m1, m2, d);
      else scan_sub<K, SHARED, false>(xs, ys, sh, r0, pl, ql, r1, r2, m1, m2, d);
    }
  }
  else {
#pragma unroll 1
    for (int r = 0; r < rows; r += 2) {
      double2 xv[K], yv[K];
#pragma unroll
      for (int k = 0; k < K; ++k) {
        xv[k] = *(const double2 *)(xs[k] + r);
        yv[k] = *(const double2 *)(ys[k] + r);
      }
      scan_rows2<K, true, false>(xv, yv, r, rows, pl, ql, r1, r2, m1, m2, d);
    }
  }
}

template <int SHARED, bool FULL>
__device__ __forceinline__ void scan_chunk_kw(int kw, const double *const *xs, const double *const *ys, const double *sh,
                                              const int *pl, const int *ql, const double *r1, const double *r2,
                                              const double *m1, const double *m2, double *d, int rows,
                                              unsigned long long touch)
{
  if (kw == 4) scan_chunk<4, SHARED, FULL>(xs, ys, sh, pl, ql, r1, r2, m1, m2, d, rows, touch);
  else if (kw == 3) scan_chunk<3, SHARED, FULL>(xs, ys, sh, pl, ql, r1, r2, m1, m2, d, rows, touch);
  else if (kw == 2) scan_chunk<2, SHARED, FULL>(xs, ys, sh, pl, ql, r1, r2, m1, m2, d, rows, touch);
  else if (kw == 1) scan_chunk<1, SHARED, FULL>(xs, ys, sh, pl, ql, r1, r2, m1, m2, d, rows, touch);
}

#define SCAN_THREADS 256
#define SCAN_STAGES 3

// one sign-class tile: tile (ti, tj) holds the pairs of the "+" vertices
// plus[32 ti .. 32 ti + 31] with the "-" vertices minus[32 tj .. 32 tj + 31], all of
// them hyperbolic (up to 1024, 4 per thread).  First the 2x2 HSVDs of DMAGF2H (the scan
// parameters of the pairs that need the column scan, compacted into shared memory that
// the row buffer reuses once every thread holds its own pairs' parameters; the other
// weights straight to W), then the tile's 64 columns stream through a three-stage
// buffer in row chunks and every thread runs its pairs' fma chains.  Only the 32-row
// sub-blocks of a chunk that hold a row p or q of some pair of the warp run the per-row
// skip test, and a warp whose pairs all have the same orientation loads the column its
// thread's pairs share once per row pair.
__global__ void __launch_bounds__(SCAN_THREADS, 2)
k_hyp_pm(const State *st, const double *__restrict__ A, const int *__restrict__ plus, const int *__restrict__ minus,
         int n_plus, int n_minus, int n, double *__restrict__ Wm)
{
  if (st->stop || st->learned_step) return;  // a learned step ranks these pairs by the scorer
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int TM = (n_minus + TW - 1) / TW;
  const int P0 = (blockIdx.x / TM) * TW, Q0 = (blockIdx.x % TM) * TW;
  HypPar *tpar = (HypPar *)smem_raw;  // [TW * TW], before the row buffer takes the space
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  __shared__ int s_cnt, s_warp[SCAN_THREADS / 32], s_col[2 * TW];
  if (tid < 2 * TW) {
    const int c = tid;
    s_col[c] = (c < TW) ? ((P0 + c < n_plus) ? plus[P0 + c] : -1) : ((Q0 + c - TW < n_minus) ? minus[Q0 + c - TW] : -1);
  }
  if (tid == 0) s_cnt = 0;
  __syncthreads();
  for (int base = 0; base < TW * TW; base += SCAN_THREADS) {
    const int l = base + tid;
    const int ci = l / TW, cj = TW + l % TW;  // tile columns of the "+" and the "-" vertex
    const int a = s_col[ci], b = s_col[cj];
    const bool valid = (a >= 0) && (b >= 0);
    const unsigned m = __ballot_sync(0xFFFFFFFFu, valid);
    if (!lane) s_warp[warp] = __popc(m);
    __syncthreads();
    int off = s_cnt;
    for (int w2 = 0; w2 < warp; ++w2) off += s_warp[w2];
    const int slot = off + __popc(m & ((1u << lane) - 1u));
    __syncthreads();
    if (tid == 0) { int t = 0; for (int w2 = 0; w2 < SCAN_THREADS / 32; ++w2) t += s_warp[w2]; s_cnt += t; }
    if (valid) {
      int pp, qq;
      bool ap;
      double w, d0 = 0.0;
      Rot t;
      const bool sc = hyp_pair_setup(A, n, a, b, pp, qq, ap, w, d0, t);
      HypPar h;
      h.p = pp; h.q = qq;
      h.pad = ap ? (ci | (cj << 8)) : (cj | (ci << 8));  // the tile columns of p and of q
      h.flags = sc ? (1 | (t.c1 ? 2 : 0) | (t.c2 ? 4 : 0)) : 0;
      h.r1 = sc ? t.r1 : 0.0; h.r2 = sc ? t.r2 : 0.0; h.m1 = sc ? t.m1 : 0.0; h.m2 = sc ? t.m2 : 0.0;
      h.d = d0;
      tpar[slot] = h;
      if (!sc) {
        if (w < -JK_HUGE) w = nan_w();
        Wm[(long long)qq * n + pp] = w;
        Wm[(long long)pp * n + qq] = w;
      }
    }
    __syncthreads();
  }
  const int cnt = s_cnt;
  if (!cnt) return;

  double *buf = (double *)smem_raw;  // [SCAN_STAGES][2 * TW][SCAN_RS]: the "+" columns, then the "-" columns
  constexpr int K = 4, STAGE = 2 * TW * SCAN_RS;
  int pv[K], qv[K], cpq[K], fl[K];  // cpq: the tile columns of p (bits 0-7) and q (bits 8-15)
  double r1[K], r2[K], m1[K], m2[K], d[K];
  int kw = 0;  // active slots of this warp (warp-uniform)
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int slot = tid + SCAN_THREADS * k;
    fl[k] = 0; pv[k] = qv[k] = -1; cpq[k] = 0; r1[k] = r2[k] = m1[k] = m2[k] = d[k] = 0.0;
    if (slot < cnt) {
      const HypPar h = tpar[slot];
      fl[k] = h.flags; pv[k] = h.p; qv[k] = h.q; cpq[k] = h.pad; d[k] = h.d;
      r1[k] = h.r1; r2[k] = h.r2; m1[k] = h.m1; m2[k] = h.m2;
    }
    if (SCAN_THREADS * k + 32 * warp < cnt) kw = k + 1;
  }
  int any = 0, fastv = 1;
  // the column layout of this thread's scanned pairs: whether p is the "+" vertex (xp)
  // and which "-" column they use (mc), if all of them agree (uni)
  int xp = -1, mc = TW;
  bool uni = true;
#pragma unroll
  for (int k = 0; k < K; ++k)
    if (fl[k] & 1) {
      any = 1;
      if ((fl[k] & 6) != 6) fastv = 0;
      const int cx = cpq[k] & 0xFF, cy = (cpq[k] >> 8) & 0xFF, isp = (cx < TW) ? 1 : 0, m = isp ? cy : cx;
      if (xp < 0) { xp = isp; mc = m; }
      else if (xp != isp || mc != m) uni = false;
    }
  // SHARED 1: every scanned pair of the warp has p = its "+" vertex and one "-" column
  // per thread, so that column is every pair's q column; SHARED 2: the "-" vertex is p
  // (with J's signs in a random permutation, only tiles near the diagonal mix the two)
  const int shared = __all_sync(0xFFFFFFFFu, uni && xp != 0) ? 1 : (__all_sync(0xFFFFFFFFu, uni && xp != 1) ? 2 : 0);
  // (this barrier also ends every read of tpar before the row buffer overwrites it)
  if (!__syncthreads_or(any)) return;
  const bool allfast = __syncthreads_and(fastv);
  const int nchunk = (n + SCAN_ROWS - 1) / SCAN_ROWS;
  // staging: this thread copies row (tid & 63) of columns (tid >> 6) + 4 j, j = 0..15
  const int sr = tid & (SCAN_ROWS - 1), sc0 = tid >> 6;
  auto stage = [&](int c) {
    if (c < nchunk) {
      double *dst = buf + (c % SCAN_STAGES) * STAGE;
      const int i0 = c * SCAN_ROWS;
      if (i0 + sr < n) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = sc0 + 4 * j;
          const int g = s_col[col];
          if (g >= 0) cp_async8(dst + col * SCAN_RS + sr, A + (long long)g * n + i0 + sr);
        }
      }
    }
    cp_async_commit();  // an empty group past the last chunk keeps the wait count uniform
  };
  stage(0);
  stage(1);
  for (int c = 0; c < nchunk; ++c) {
    cp_async_wait<1>();  // chunk c has landed (chunk c + 1 may be in flight)
    __syncthreads();     // ... for every thread; and everyone is done with chunk c - 1
    stage(c + 2);        // into the buffer of chunk c - 1
    const double *bb = buf + (c % SCAN_STAGES) * STAGE;
    const int i0 = c * SCAN_ROWS, rows = min(SCAN_ROWS, n - i0);
    const double *xs[K], *ys[K];
    int pr[K], qr[K];
    unsigned long long mine = 0;  // the chunk's rows that are p or q of this thread's scanned pairs
#pragma unroll
    for (int k = 0; k < K; ++k) {
      xs[k] = bb + (cpq[k] & 0xFF) * SCAN_RS;
      ys[k] = bb + ((cpq[k] >> 8) & 0xFF) * SCAN_RS;
      pr[k] = pv[k] - i0;  // p, q as rows of this chunk
      qr[k] = qv[k] - i0;
      if (fl[k] & 1) {
        if (pr[k] >= 0 && pr[k] < rows) mine |= 1ull << pr[k];
        if (qr[k] >= 0 && qr[k] < rows) mine |= 1ull << qr[k];
      }
    }
    if (allfast) {
      const unsigned long long touch =
          (unsigned long long)__reduce_or_sync(0xFFFFFFFFu, (unsigned)mine) |
          ((unsigned long long)__reduce_or_sync(0xFFFFFFFFu, (unsigned)(mine >> 32)) << 32);
      const double *sh = bb + mc * SCAN_RS;
      if (rows == SCAN_ROWS) {
        if (shared == 1) scan_chunk_kw<1, true>(kw, xs, ys, sh, pr, qr, r1, r2, m1, m2, d, rows, touch);
        else if (shared == 2) scan_chunk_kw<2, true>(kw, xs, ys, sh, pr, qr, r1, r2, m1, m2, d, rows, touch);
        else scan_chunk_kw<0, true>(kw, xs, ys, sh, pr, qr, r1, r2, m1, m2, d, rows, touch);
      }
      else {
        if (shared == 1) scan_chunk_kw<1, false>(kw, xs, ys, sh, pr, qr, r1, r2, m1, m2, d, rows, touch);
        else if (shared == 2) scan_chunk_kw<2, false>(kw, xs, ys, sh, pr, qr, r1, r2, m1, m2, d, rows, touch);
        else scan_chunk_kw<0, false>(kw, xs, ys, sh, pr, qr, r1, r2, m1, m2, d, rows, touch);
      }
    }
    else {
#pragma unroll
      for (int k = 0; k < K; ++k)
        if (fl[k] & 1) {
          Rot t;
          t.c1 = (fl[k] >> 1) & 1; t.c2 = (fl[k] >> 2) & 1;
          t.r1 = r1[k]; t.r2 = r2[k]; t.m1 = m1[k]; t.m2 = m2[k];
          scan_rows_real(xs[k], ys[k], rows, i0, pv[k], qv[k], t, d[k]);
        }
    }
  }
  cp_async_wait<0>();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    if (!(fl[k] & 1)) continue;
    const int p = pv[k], q = qv[k];
    double x = d[k];
    if (x < -JK_HUGE) x = nan_w();
    Wm[(long long)q * n + p] = x;
    Wm[(long long)p * n + q] = x;
  }
}

// |A(i,j)| of every entry of a complex A (the project's hypot), once per step: the
// column scan of ABODNZF2 needs the magnitude of every unrotated entry of its two
// columns, and every pair of a column would otherwise compute it again
__global__ void k_absmat(const State *st, const double2 *__restrict__ A, long long nn, double *__restrict__ mag)
{
  if (st->stop || st->learned_step) return;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nn; k += (long long)gridDim.x * blockDim.x)
    mag[k] = zabs(A[k]);
}

// ABODNZF2's row scan (src/Z/ztransf.F90:452-637) with the magnitudes of the unrotated
// entries taken from xa, ya: the same operations in the same order as scan_rows_cplx
__device__ __forceinline__ void scan_rows_cplx_mag(const double2 *xs, const double2 *ys, const double *xa, const double *ya,
                                                   int rows, int i0, int p, int q, const ZRot &t, double &d)
{
  for (int r = 0; r < rows; ++r) {
    double2 x = xs[r], y = ys[r];
    zrot_apply_ab(t, x, y);
    const int i = i0 + r;
    if (i != p && i != q) {
      const double axi = xa[r], axx = zabs(x), ayi = ya[r], ayy = zabs(y);
      d = fma(__dsub_rn(axi, axx), __dadd_rn(axi, axx), d);
      d = fma(__dsub_rn(ayi, ayy), __dadd_rn(ayi, ayy), d);
    }
  }
}

// The complex hyperbolic weights (ZMAGF2H, src/Z/zstep.F90:43-74): the tile of
// k_weights_hyp with the unrotated magnitudes staged beside the columns (48 rows per
// chunk to stay within the static shared-memory limit)
#define ZHR 48
template <int HP, int HM>
__global__ void __launch_bounds__(HP * HM)
k_weights_hyp_z(const State *st, const double2 *__restrict__ A, const double *__restrict__ mag, const int *__restrict__ plus,
                const int *__restrict__ minus, int n_plus, int n_minus, double *__restrict__ Wm, int n)
{
  if (st->stop || st->learned_step) return;  // a learned step ranks these pairs by the scorer
  __shared__ double2 sP[HP][ZHR + 1];
  __shared__ double2 sM[HM][ZHR + 1];
  __shared__ double aP[HP][ZHR + 1];
  __shared__ double aM[HM][ZHR + 1];
  const int tx = threadIdx.x % HP, ty = threadIdx.x / HP;
  const int ia = blockIdx.x * HP + tx, ib = blockIdx.y * HM + ty;
  const bool valid = (ia < n_plus) && (ib < n_minus);
  int p = 0, q = 0;
  bool scan = false, a_is_p = true;
  double d = 0.0, w = nan_w();
  ZRot t;
  if (valid) {
    const int a = plus[ia], b = minus[ib];
    a_is_p = (a < b);
    p = a_is_p ? a : b;
    q = a_is_p ? b : a;
    const double2 app = A[(long long)p * n + p], aqp = A[(long long)p * n + q], apq = A[(long long)q * n + p],
                  aqq = A[(long long)q * n + q];
    if (may_transform(app, aqp, apq, aqq)) {
      double2 A2[4] = { app, aqp, apq, aqq }, U2[4], Z2[4];
      int info = 0;
      const int jp = a_is_p ? 1 : -1;  // "+" column a, "-" column b
      zhsvd2(A2, jp, -jp, U2, Z2, JK_TH1FIX, info);
      if (info < 0) w = nan_w();
      else if (!(info & 1)) w = 0.0;
      else if (!(info & 4)) w = dasum4(aqp.x, aqp.y, apq.x, apq.y);
      else {
        // the two off-diagonal terms that start ABODNZF2
        const double2 a1 = (info & 8) ? A2[M21] : make_double2(0.0, 0.0);
        const double2 a2 = (info & 8) ? A2[M12] : make_double2(0.0, 0.0);
        d = 0.0;
        d = fma(__dsub_rn(aqp.x, a1.x), __dadd_rn(aqp.x, a1.x), d);
        d = fma(__dsub_rn(aqp.y, a1.y), __dadd_rn(aqp.y, a1.y), d);
        d = fma(__dsub_rn(apq.x, a2.x), __dadd_rn(apq.x, a2.x), d);
        d = fma(__dsub_rn(apq.y, a2.y), __dadd_rn(apq.y, a2.y), d);
        t = zrot_ab(Z2);
        scan = true;
      }
    }
  }
  if (!__syncthreads_or(scan)) {
    if (valid) {
      if (w < -JK_HUGE) w = nan_w();
      Wm[(long long)q * n + p] = w;
      Wm[(long long)p * n + q] = w;
    }
    return;
  }
  const int pa = blockIdx.x * HP, pb = blockIdx.y * HM;
  for (int i0 = 0; i0 < n; i0 += ZHR) {
    const int rows = min(ZHR, n - i0);
    for (int k = threadIdx.x; k < (HP + HM) * ZHR; k += HP * HM) {
      const int c = k / ZHR, r = k % ZHR;
      if (r < rows) {
        if (c < HP) {
          const int ca = pa + c;
          if (ca < n_plus) {
            const long long g = (long long)plus[ca] * n + i0 + r;
            sP[c][r] = A[g];
            aP[c][r] = mag[g];
          }
        }
        else {
          const int cb = pb + (c - HP);
          if (cb < n_minus) {
            const long long g = (long long)minus[cb] * n + i0 + r;
            sM[c - HP][r] = A[g];
            aM[c - HP][r] = mag[g];
          }
        }
      }
    }
    __syncthreads();
    if (scan) {
      const double2 *xs = a_is_p ? sP[tx] : sM[ty];
      const double2 *ys = a_is_p ? sM[ty] : sP[tx];
      const double *xa = a_is_p ? aP[tx] : aM[ty];
      const double *ya = a_is_p ? aM[ty] : aP[tx];
      scan_rows_cplx_mag(xs, ys, xa, ya, rows, i0, p, q, t, d);
    }
    __syncthreads();
  }
  if (valid) {
    if (scan) w = d;
    if (w < -JK_HUGE) w = nan_w();
    Wm[(long long)q * n + p] = w;
    Wm[(long long)p * n + q] = w;
  }
}

// The complex hyperbolic weights, pipelined (k_hyp_z_pm below): sign-class tiles of 16
// "+" by 32 "-" vertices (512 pairs, two per thread), 32 rows per chunk of the columns
// and of their unrotated magnitudes staged with cp.async in two buffers, the sequential
// ABODNZF2 chains of the two pairs of a thread interleaved.
#define ZTP 16
#define ZTM 32
#define ZTC (ZTP + ZTM)
#define ZROWS 32
#define ZRS (ZROWS + 1)  // padded column: the 16-byte (8-byte) reads of a warp hit distinct banks
#define ZSTAGES 2
#define ZTHREADS 256
constexpr size_t kZStage = (size_t)ZTC * ZRS * (sizeof(double2) + sizeof(double));
constexpr size_t kZSmem = ZSTAGES * kZStage;

// scan parameters of one complex hyperbolic pair
struct ZHypPar {
  double2 r1, r2, m1, m2;  // the AB coefficients of Z2
  double d;                // the four leading terms
  int p, q;                // the pair (0-based, p < q)
  int flags;               // bit0 scan, bit1 c1, bit2 c2
  int cols;                // the tile columns of p (bits 0-7) and q (bits 8-15)
};
static_assert(ZTP * ZTM * sizeof(ZHypPar) <= kZSmem, "a tile's scan parameters must fit in the row buffer");

// hypot2 out of line: the rare operands hypot2_fast does not take
__device__ __noinline__ double hypot2_call(double x, double y) { return hypot2(x, y); }

// (the range test is repeated inside hypot2_fast; a form that tests once, with the fast path
// split out, measured 2% slower in k_hyp_z_pm: more registers spilled)
__device__ __forceinline__ double zabs_scan(double2 a)
{
  const double ax = fabs(a.x), ay = fabs(a.y);
  const double u = (ax >= ay) ? ax : ay;
  const double v = (ax >= ay) ? ay : ax;
  const int bu = (int)((unsigned long long)__double_as_longlong(u) >> 52);
  const int bv = (int)((unsigned long long)__double_as_longlong(v) >> 52);
  if (bu >= 23 && bu <= 2021 && bv >= 1 && ax == ax && ay == ay) return hypot2_fast(a.x, a.y);
  return hypot2_call(a.x, a.y);
}

// rows 0 .. rows - 1 of a chunk for K pairs per thread (ABODNZF2, src/Z/ztransf.F90:452-637:
// the rotation, then the magnitudes of the rotated and of the unrotated entries, rows p and
// q skipped).  FAST: every pair of the block takes the first branch (c1, c2); otherwise
// each pair selects its branches.  Slots without a scan compute nothing.
template <int K, bool FAST>
__device__ __forceinline__ void zscan_rows(const double2 *const *xs, const double2 *const *ys, const double *const *xa,
                                           const double *const *ya, int rows, const int *pl, const int *ql,
                                           const int *fl, const ZRot *t, double *d)
{
#pragma unroll 1
  for (int r = 0; r < rows; ++r) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!(fl[k] & 1)) continue;
      double2 x = xs[k][r], y = ys[k][r];
      if (FAST) {
        const double2 xx = zzfma(y, t[k].r1, x), yy = zzfma(x, t[k].r2, y);
        x = zzmul(xx, t[k].m1);
        y = zzmul(yy, t[k].m2);
      }
      else zrot_apply_ab(t[k], x, y);
      if (r != pl[k] && r != ql[k]) {
        const double axi = xa[k][r], axx = zabs_scan(x), ayi = ya[k][r], ayy = zabs_scan(y);
        d[k] = fma(__dsub_rn(axi, axx), __dadd_rn(axi, axx), d[k]);
        d[k] = fma(__dsub_rn(ayi, ayy), __dadd_rn(ayi, ayy), d[k]);
      }
    }
  }
}

// one complex sign-class tile: tile t holds the pairs of the "+" vertices plus[16 (t / TM) ..]
// with the "-" vertices minus[32 (t % TM) ..] (TM tiles of "-" vertices), all hyperbolic.
// First the 2x2 HSVDs of ZMAGF2H (src/Z/zstep.F90:43-74; the scan parameters of the pairs
// that need the column scan, compacted into the shared memory the row buffer takes over
// once every thread holds its own pairs' parameters; the other weights straight to W), then
// the tile's 48 columns and their magnitudes stream through two buffers in row chunks.
__global__ void __launch_bounds__(ZTHREADS, 2)
k_hyp_z_pm(const State *st, const double2 *__restrict__ A, const double *__restrict__ mag, const int *__restrict__ plus,
           const int *__restrict__ minus, int n_plus, int n_minus, int n, double *__restrict__ Wm)
{
  if (st->stop || st->learned_step) return;  // a learned step ranks these pairs by the scorer
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int TM = (n_minus + ZTM - 1) / ZTM;
  const int P0 = (blockIdx.x / TM) * ZTP, Q0 = (blockIdx.x % TM) * ZTM;
  ZHypPar *tpar = (ZHypPar *)smem_raw;  // [ZTP * ZTM], before the row buffer takes the space
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  __shared__ int s_cnt, s_warp[ZTHREADS / 32], s_col[ZTC];
  if (tid < ZTC) {
    const int c = tid;
    s_col[c] = (c < ZTP) ? ((P0 + c < n_plus) ? plus[P0 + c] : -1) : ((Q0 + c - ZTP < n_minus) ? minus[Q0 + c - ZTP] : -1);
  }
  if (tid == 0) s_cnt = 0;
  __syncthreads();
  for (int base = 0; base < ZTP * ZTM; base += ZTHREADS) {
    const int l = base + tid;
    const int ci = l / ZTM, cj = ZTP + l % ZTM;  // tile columns of the "+" and the "-" vertex
    const int a = s_col[ci], b = s_col[cj];
    const bool valid = (a >= 0) && (b >= 0);
    const unsigned m = __ballot_sync(0xFFFFFFFFu, valid);
    if (!lane) s_warp[warp] = __popc(m);
    __syncthreads();
    int off = s_cnt;
    for (int w2 = 0; w2 < warp; ++w2) off += s_warp[w2];
    const int slot = off + __popc(m & ((1u << lane) - 1u));
    __syncthreads();
    if (tid == 0) { int t = 0; for (int w2 = 0; w2 < ZTHREADS / 32; ++w2) t += s_warp[w2]; s_cnt += t; }
    if (valid) {
      const bool ap = (a < b);
      const int p = ap ? a : b, q = ap ? b : a;
      const double2 app = A[(long long)p * n + p], aqp = A[(long long)p * n + q], apq = A[(long long)q * n + p],
                    aqq = A[(long long)q * n + q];
      ZHypPar h;
      h.p = p; h.q = q;
      h.cols = ap ? (ci | (cj << 8)) : (cj | (ci << 8));
      h.flags = 0;
      h.d = 0.0;
      h.r1 = h.r2 = h.m1 = h.m2 = make_double2(0.0, 0.0);
      double w = nan_w();
      if (may_transform(app, aqp, apq, aqq)) {
        double2 A2[4] = { app, aqp, apq, aqq }, U2[4], Z2[4];
        int info = 0;
        const int jp = ap ? 1 : -1;  // "+" column a, "-" column b
        zhsvd2(A2, jp, -jp, U2, Z2, JK_TH1FIX, info);
        if (info < 0) w = nan_w();
        else if (!(info & 1)) w = 0.0;
        else if (!(info & 4)) w = dasum4(aqp.x, aqp.y, apq.x, apq.y);
        else {
          // the four off-diagonal terms that start ABODNZF2
          const double2 a1 = (info & 8) ? A2[M21] : make_double2(0.0, 0.0);
          const double2 a2 = (info & 8) ? A2[M12] : make_double2(0.0, 0.0);
          double d = 0.0;
          d = fma(__dsub_rn(aqp.x, a1.x), __dadd_rn(aqp.x, a1.x), d);
          d = fma(__dsub_rn(aqp.y, a1.y), __dadd_rn(aqp.y, a1.y), d);
          d = fma(__dsub_rn(apq.x, a2.x), __dadd_rn(apq.x, a2.x), d);
          d = fma(__dsub_rn(apq.y, a2.y), __dadd_rn(apq.y, a2.y), d);
          const ZRot t = zrot_ab(Z2);
          h.r1 = t.r1; h.r2 = t.r2; h.m1 = t.m1; h.m2 = t.m2;
          h.flags = 1 | (t.c1 ? 2 : 0) | (t.c2 ? 4 : 0);
          h.d = d;
        }
      }
      tpar[slot] = h;
      if (!(h.flags & 1)) {
        if (w < -JK_HUGE) w = nan_w();
        Wm[(long long)q * n + p] = w;
        Wm[(long long)p * n + q] = w;
      }
    }
    __syncthreads();
  }
  const int cnt = s_cnt;
  if (!cnt) return;

  double2 *bz = (double2 *)smem_raw;                                          // [ZSTAGES][ZTC][ZRS]
  double *bm = (double *)(smem_raw + ZSTAGES * ZTC * ZRS * sizeof(double2));  // [ZSTAGES][ZTC][ZRS]
  constexpr int K = 2, STAGE = ZTC * ZRS;
  int pv[K], qv[K], cpq[K], fl[K];
  ZRot t[K];
  double d[K];
  int kw = 0;  // active slots of this warp (warp-uniform)
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int slot = tid + ZTHREADS * k;
    fl[k] = 0; pv[k] = qv[k] = -1; cpq[k] = 0; d[k] = 0.0;
    t[k].r1 = t[k].r2 = t[k].m1 = t[k].m2 = make_double2(0.0, 0.0);
    t[k].c1 = t[k].c2 = 1;
    if (slot < cnt) {
      const ZHypPar h = tpar[slot];
      fl[k] = h.flags; pv[k] = h.p; qv[k] = h.q; cpq[k] = h.cols; d[k] = h.d;
      t[k].r1 = h.r1; t[k].r2 = h.r2; t[k].m1 = h.m1; t[k].m2 = h.m2;
      t[k].c1 = (h.flags >> 1) & 1; t[k].c2 = (h.flags >> 2) & 1;
    }
    if (ZTHREADS * k + 32 * warp < cnt) kw = k + 1;
  }
  int any = 0, fastv = 1;
#pragma unroll
  for (int k = 0; k < K; ++k)
    if (fl[k] & 1) { any = 1; if ((fl[k] & 6) != 6) fastv = 0; }
  // (this barrier also ends every read of tpar before the row buffer overwrites it)
  if (!__syncthreads_or(any)) return;
  const bool allfast = __syncthreads_and(fastv);
  const int nchunk = (n + ZROWS - 1) / ZROWS;
  auto stage = [&](int c) {
    if (c < nchunk) {
      double2 *dz = bz + (c % ZSTAGES) * STAGE;
      double *dm = bm + (c % ZSTAGES) * STAGE;
      const int i0 = c * ZROWS;
#pragma unroll
      for (int j = 0; j < (ZTC * ZROWS) / ZTHREADS; ++j) {
        const int idx = tid + ZTHREADS * j, col = idx / ZROWS, r = idx % ZROWS;
        const int g = s_col[col];
        if (g >= 0 && i0 + r < n) {
          const long long e = (long long)g * n + i0 + r;
          cp_async16(dz + col * ZRS + r, A + e);
          cp_async8(dm + col * ZRS + r, mag + e);
        }
      }
    }
    cp_async_commit();  // an empty group past the last chunk keeps the wait count uniform
  };
  static_assert((ZTC * ZROWS) % ZTHREADS == 0, "the staging copies divide among the threads");
  stage(0);
  for (int c = 0; c < nchunk; ++c) {
    stage(c + 1);        // into the buffer of chunk c - 1, which every thread is done with
    cp_async_wait<1>();  // chunk c has landed (chunk c + 1 may be in flight)
    __syncthreads();
    const double2 *cz = bz + (c % ZSTAGES) * STAGE;
    const double *cm = bm + (c % ZSTAGES) * STAGE;
    const int i0 = c * ZROWS, rows = min(ZROWS, n - i0);
    const double2 *xs[K], *ys[K];
    const double *xa[K], *ya[K];
    int pr[K], qr[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int cx = cpq[k] & 0xFF, cy = (cpq[k] >> 8) & 0xFF;
      xs[k] = cz + cx * ZRS; ys[k] = cz + cy * ZRS;
      xa[k] = cm + cx * ZRS; ya[k] = cm + cy * ZRS;
      pr[k] = pv[k] - i0;  // p, q as rows of this chunk
      qr[k] = qv[k] - i0;
    }
    if (allfast) {
      if (kw == 2) zscan_rows<2, true>(xs, ys, xa, ya, rows, pr, qr, fl, t, d);
      else if (kw == 1) zscan_rows<1, true>(xs, ys, xa, ya, rows, pr, qr, fl, t, d);
    }
    else {
      if (kw == 2) zscan_rows<2, false>(xs, ys, xa, ya, rows, pr, qr, fl, t, d);
      else if (kw == 1) zscan_rows<1, false>(xs, ys, xa, ya, rows, pr, qr, fl, t, d);
    }
    __syncthreads();  // every thread is done with chunk c before chunk c + 2 overwrites it
  }
  cp_async_wait<0>();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    if (!(fl[k] & 1)) continue;
    const int p = pv[k], q = qv[k];
    double x = d[k];
    if (x < -JK_HUGE) x = nan_w();
    Wm[(long long)q * n + p] = x;
    Wm[(long long)p * n + q] = x;
  }
}

template <typename T, int HP, int HM>
__global__ void __launch_bounds__(HP * HM)
k_weights_hyp(const State *st, const T *__restrict__ A, const int *__restrict__ plus, const int *__restrict__ minus,
              int n_plus, int n_minus, double *__restrict__ Wm, int n)
{
  if (st->stop || st->learned_step) return;  // a learned step ranks these pairs by the scorer
  __shared__ T sP[HP][HR + 1];
  __shared__ T sM[HM][HR + 1];
  const int tx = threadIdx.x % HP, ty = threadIdx.x / HP;
  const int ia = blockIdx.x * HP + tx, ib = blockIdx.y * HM + ty;
  const bool valid = (ia < n_plus) && (ib < n_minus);
  int p = 0, q = 0;
  bool scan = false, a_is_p = true;
  double d = 0.0, w = nan_w();
  typename Tr<T>::R t;
  if (valid) {
    const int a = plus[ia], b = minus[ib];
    a_is_p = (a < b);
    p = a_is_p ? a : b;
    q = a_is_p ? b : a;
    const T app = A[(long long)p * n + p], aqp = A[(long long)p * n + q], apq = A[(long long)q * n + p], aqq = A[(long long)q * n + q];
    if (may_transform(app, aqp, apq, aqq)) {
      T A2[4] = { app, aqp, apq, aqq }, U2[4], Z2[4];
      int info = 0;
      const int jp = a_is_p ? 1 : -1;  // "+" column a, "-" column b
      Tr<T>::hsvd2(A2, jp, -jp, U2, Z2, JK_TH1FIX, info);
      if (info < 0) w = nan_w();
      else if (!(info & 1)) w = 0.0;
      else if (!(info & 4)) w = Tr<T>::magt(aqp, apq);
      else {
        // the two off-diagonal terms that start ABODNDF2 / ABODNZF2
        const T aqp2 = (info & 8) ? A2[M21] : Tr<T>::zero();
        const T apq2 = (info & 8) ? A2[M12] : Tr<T>::zero();
        if constexpr (sizeof(T) == sizeof(double)) {
          const double xq = *(const double *)&aqp, yp = *(const double *)&apq;
          const double a1 = *(const double *)&aqp2, a2 = *(const double *)&apq2;
          d = 0.0;
          d = fma(__dsub_rn(xq, a1), __dadd_rn(xq, a1), d);
          d = fma(__dsub_rn(yp, a2), __dadd_rn(yp, a2), d);
        }
        else {
          const double2 xq = *(const double2 *)&aqp, yp = *(const double2 *)&apq;
          const double2 a1 = *(const double2 *)&aqp2, a2 = *(const double2 *)&apq2;
          d = 0.0;
          d = fma(__dsub_rn(xq.x, a1.x), __dadd_rn(xq.x, a1.x), d);
          d = fma(__dsub_rn(xq.y, a1.y), __dadd_rn(xq.y, a1.y), d);
          d = fma(__dsub_rn(yp.x, a2.x), __dadd_rn(yp.x, a2.x), d);
          d = fma(__dsub_rn(yp.y, a2.y), __dadd_rn(yp.y, a2.y), d);
        }
        t = Tr<T>::ab(Z2);
        scan = true;
      }
    }
  }
  // a block-uniform exit when no thread of the tile scans
  if (!__syncthreads_or(scan)) {
    if (valid) {
      if (w < -JK_HUGE) w = nan_w();
      Wm[(long long)q * n + p] = w;
      Wm[(long long)p * n + q] = w;
    }
    return;
  }
  const int pa = blockIdx.x * HP, pb = blockIdx.y * HM;
  for (int i0 = 0; i0 < n; i0 += HR) {
    const int rows = min(HR, n - i0);
    // stage rows [i0, i0+rows) of the tile's HP + HM columns
    for (int k = threadIdx.x; k < (HP + HM) * HR; k += HP * HM) {
      const int c = k / HR, r = k % HR;
      if (r < rows) {
        if (c < HP) {
          const int ca = pa + c;
          if (ca < n_plus) sP[c][r] = A[(long long)plus[ca] * n + i0 + r];
        }
        else {
          const int cb = pb + (c - HP);
          if (cb < n_minus) sM[c - HP][r] = A[(long long)minus[cb] * n + i0 + r];
        }
      }
    }
    __syncthreads();
    if (scan) {
      const T *xs = a_is_p ? sP[tx] : sM[ty];
      const T *ys = a_is_p ? sM[ty] : sP[tx];
      if constexpr (sizeof(T) == sizeof(double)) scan_rows_real((const double *)xs, (const double *)ys, rows, i0, p, q, *(const Rot *)&t, d);
      else scan_rows_cplx((const double2 *)xs, (const double2 *)ys, rows, i0, p, q, *(const ZRot *)&t, d);
    }
    __syncthreads();
  }
  if (valid) {
    if (scan) w = d;
    if (w < -JK_HUGE) w = nan_w();
    Wm[(long long)q * n + p] = w;
    Wm[(long long)p * n + q] = w;
  }
}

// ---------------------------------------------------------------------------
// selection: the greedy non-colliding pivots of the sorted record list
// (AW_SRT1/2 + AW_NCP1/2, src/shared/atypes.F90:85-484)
//
// The records are ordered by descending weight, then descending band q-p, then
// descending p (AW_CMP).  Walking them in that order and taking every record whose
// p and q are both unused is the greedy matching of the weighted graph.  The walk
// stops after N_2 records: those are the N_2 highest-ranked edges of the full
// greedy matching, so the matched edges are ranked and the first N_2 kept, in rank
// order (the STEP array).
//
// The matching is built in rounds: every free vertex proposes to its best free
// partner and mutual proposals are matched; the best remaining edge of both its
// endpoints is always taken by the walk, so the rounds rebuild the walk's matching
// without touching the record list.  k_colsort ranks every vertex's partners once
// per step (one block per column of the symmetric weight matrix; a bitonic sort held
// in registers, shuffles and shared memory), so a round only moves each free
// vertex's list pointer past partners matched meanwhile (k_select, one block).
// ---------------------------------------------------------------------------
#ifndef SEL_THREADS
#define SEL_THREADS 1024  // threads of the one-block selection (a tuning knob)
#endif
#define SORT_THREADS 256
#ifndef JK_SEL_CLUSTER_MIN_N
#define JK_SEL_CLUSTER_MIN_N 512  // the cluster matching from this order on (a tuning knob)
#endif
constexpr int kSelClusterMinN = JK_SEL_CLUSTER_MIN_N;

// descending bitonic sort of s2 (a power of two) records (k, t, i) in shared memory
__device__ __forceinline__ void bitonic_desc(unsigned long long *k, unsigned *t, int *ix, int s2)
{
  for (int kk = 2; kk <= s2; kk <<= 1)
    for (int j = kk >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < s2; i += blockDim.x) {
        const int l = i ^ j;
        if (l > i) {
          const bool desc = ((i & kk) == 0);
          const bool lbetter = kbetter(k[l], t[l], k[i], t[i]);
          if (desc == lbetter) {
            const unsigned long long a = k[i]; k[i] = k[l]; k[l] = a;
            const unsigned b = t[i]; t[i] = t[l]; t[l] = b;
            const int c = ix[i]; ix[i] = ix[l]; ix[l] = c;
          }
        }
      }
      __syncthreads();
    }
}

__host__ __device__ __forceinline__ int pow2ceil(int x)
{
  int s = 1;
  while (s < x) s <<= 1;
  return s;
}

// list row stride: 8 entries (16 bytes) per vector load
__host__ __device__ __forceinline__ int list_ld(int n) { return (n + 7) & ~7; }

// rank the partners of vertex v = blockIdx.x: list[v][r] = r-th best partner,
// rank[v][u] = position of u in that list, len[v] = number of partners.
// One 64-bit key per partner: the top 48 bits of the weight key, then the 16-bit
// tie code (band << 1 | (u > v)), which orders the partners of v as (band, p) do
// and also names u.  Partners whose keys agree in the top 48 bits are re-ordered by
// the full key afterwards.  E keys per thread in registers (position tid*E + e);
// stages with partner distance < E run in registers, < 32E by warp shuffles, the
// rest in shared memory.
__device__ __forceinline__ unsigned long long ckey(double w, int u, int v)
{
  const unsigned long long k = wkey(w);
  if (!k) return 0ULL;
  const unsigned b = (unsigned)((u < v) ? (v - u) : (u - v));
  return ((k >> 16) << 16) | (unsigned long long)((b << 1) | (u > v ? 1u : 0u));
}

__device__ __forceinline__ int ckey_u(unsigned long long c, int v)
{
  const int t = (int)(c & 0xFFFFu);
  return (t & 1) ? v + (t >> 1) : v - (t >> 1);
}

// descending bitonic sort of the SORT_THREADS * E keys a block holds E per thread
// (position tid * E + e): stages with partner distance < E in registers, < 32 E by warp
// shuffles, the rest through shared memory (sk, SORT_THREADS * E entries)
template <int E>
__device__ __forceinline__ void block_sort_desc(unsigned long long (&k)[E], unsigned long long *sk)
{
  const int tid = threadIdx.x, s2 = SORT_THREADS * E;
  for (int kk = 2; kk <= s2; kk <<= 1) {
    for (int j = kk >> 1; j >= E; j >>= 1) {
      if (j < 32 * E) {
        const int m = j / E;
        const bool lower = ((tid & m) == 0);
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const unsigned long long ok = __shfl_xor_sync(0xFFFFFFFFu, k[e], m);
          const bool desc = (((tid * E + e) & kk) == 0);
          // the lower position of a descending pair keeps the larger key
          const unsigned long long hi = (ok > k[e]) ? ok : k[e], lo = (ok > k[e]) ? k[e] : ok;
          k[e] = (desc == lower) ? hi : lo;
        }
      }
      else {
        __syncthreads();
#pragma unroll
        for (int e = 0; e < E; ++e) sk[tid * E + e] = k[e];
        __syncthreads();
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int i = tid * E + e, l = i ^ j;
          const unsigned long long ok = sk[l];
          const bool desc = ((i & kk) == 0), lower = (i < l);
          const unsigned long long hi = (ok > k[e]) ? ok : k[e], lo = (ok > k[e]) ? k[e] : ok;
          k[e] = (desc == lower) ? hi : lo;
        }
      }
    }
#pragma unroll
    for (int jj = E / 2; jj > 0; jj >>= 1) {
      if (jj < kk) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int f = e ^ jj;
          if (f > e) {
            const bool desc = (((tid * E + e) & kk) == 0);
            if (desc == (k[f] > k[e])) { const unsigned long long a = k[e]; k[e] = k[f]; k[f] = a; }
          }
        }
      }
    }
  }
}

template <int E>
__global__ void __launch_bounds__(SORT_THREADS)
k_colsort(const State *st, const double *__restrict__ Wm, int n, unsigned short *list, unsigned short *rank, int *len)
{
  if (st->stop) return;
  __shared__ unsigned long long sk[SORT_THREADS * E];
  __shared__ unsigned short slo[SORT_THREADS * E];  // low 16 bits of the sorted keys' weight keys
  __shared__ int s_cnt, s_warp[SORT_THREADS / 32];
  const int v = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double *col = Wm + (long long)v * n;
  unsigned long long k[E];
  int valid = 0;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int i = tid * E + e;
    k[e] = (i < n && i != v) ? ckey(col[i], i, v) : 0ULL;
    valid += k[e] ? 1 : 0;
  }
  if (tid == 0) s_cnt = 0;
  __syncthreads();
  atomicAdd(&s_cnt, valid);
  block_sort_desc<E>(k, sk);
  __syncthreads();
  const int cnt = s_cnt;
  // The sort saw the top 48 bits of each weight key: keys that agree there but differ in
  // the low 16 bits are in tie-code order and must be reordered by the full key.  The low
  // bits of every sorted key show whether any run of equal top bits needs it (near
  // convergence many weights are exactly equal, zeros above all: such runs are already in
  // the record order).
  unsigned lo[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int i = tid * E + e;
    sk[i] = k[e];
    lo[e] = (i < cnt) ? (unsigned)(wkey(col[ckey_u(k[e], v)]) & 0xFFFFu) : 0u;
    slo[i] = (unsigned short)lo[e];
  }
  __syncthreads();
  int bad = 0, starts = 0;
  bool start[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int i = tid * E + e;
    const bool same = (i > 0) && (i < cnt) && ((sk[i - 1] >> 16) == (k[e] >> 16));
    start[e] = (i < cnt) && !same;
    starts += start[e] ? 1 : 0;
    if (same && slo[i - 1] != (unsigned short)lo[e]) bad = 1;
  }
  if (__syncthreads_or(bad)) {
    // order every run by (low bits, tie code): a second sort on (run index, low 16 bits,
    // tie code), the run index from a block-wide prefix count of the run starts
    int c = starts;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xFFFFFFFFu, c, o);
      if (lane >= o) c += t;
    }
    if (lane == 31) s_warp[warp] = c;
    __syncthreads();
    if (warp == 0) {
      int x = (lane < SORT_THREADS / 32) ? s_warp[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += t;
      }
      if (lane < SORT_THREADS / 32) s_warp[lane] = x;
    }
    __syncthreads();
    int run = c - starts + (warp > 0 ? s_warp[warp - 1] : 0) - 1;  // the run before my first key
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int i = tid * E + e;
      run += start[e] ? 1 : 0;
      k[e] = (i < cnt) ? (((unsigned long long)(0xFFFFu - (unsigned)run) << 32) | ((unsigned long long)lo[e] << 16) |
                          (k[e] & 0xFFFFull))
                       : 0ULL;
    }
    block_sort_desc<E>(k, sk);  // the low 16 bits (the tie code, which names the partner) are kept
    __syncthreads();
#pragma unroll
    for (int e = 0; e < E; ++e) sk[tid * E + e] = k[e];
    __syncthreads();
  }
  unsigned short *lv = list + (long long)v * list_ld(n);
  unsigned short *rv = rank + (long long)v * n;
  for (int r = tid; r < cnt; r += blockDim.x) {
    const int u = ckey_u(sk[r], v);
    lv[r] = (unsigned short)u;
    rv[u] = (unsigned short)r;
  }
  if (tid == 0) len[v] = cnt;
}

// the end of the previous step: SL := MIN(SL, NL) and the loop test
// (src/D/dstep.F90:442, 564-583), with the statistics of DSTEP_TRANSF
// (src/D/dstep.F90:349-370) when tracing
template <typename T>
__device__ void end_of_step(State *st, const Piv<T> *piv, const int *J, Trace &tr)
{
  if (!st->pending || st->stop) return;
  st->pending = 0;
  const int sl = st->sl, nl = st->nl, err = st->err;
  if (st->trace_on) {
    double tw = -0.0;
    int tg = 0, hy = 0;
    if (err == 0)
      for (int i = 0; i < sl; ++i) {
        const int l = piv[i].info;
        if ((l & 2) || (l & 4)) {
          tw = __dadd_rn(tw, piv[i].w);
          if (J[piv[i].p] == J[piv[i].q]) ++tg; else ++hy;
        }
      }
    if (st->trace_steps < st->trace_cap_steps) {
      const int s = st->trace_steps++;
      tr.sl[s] = sl; tr.nl[s] = (err < 0) ? err : nl; tr.tw[s] = tw; tr.trig[s] = tg; tr.hyp[s] = hy;
      tr.rounds[s] = st->rounds;
    }
    for (int i = 0; i < sl; ++i)
      if (st->trace_npiv < st->trace_cap_piv) tr.piv[st->trace_npiv++] = make_int2(piv[i].p, piv[i].q);
  }
  if (err < 0) { st->info = err; st->stop = 1; }
  else if (((sl < nl) ? sl : nl) <= 0) {
    // only a step ranked by the exact weights ends the loop; a learned step without an
    // effective pivot is followed by an exact one
    if (st->retry) st->retry = 0;
    else { st->info = st->steps; st->stop = 1; }
  }
  else {
    st->steps += 1;
    // the caller's step limit: the loop waits here, between two steps, and can go on
    if (st->limit > 0 && st->steps >= st->limit) st->stop = 2;
  }
}

// The walk of one free vertex's ranked partner list from its pointer to the first free
// partner (-1: none left).  The vertex's window holds list entries wbase .. wbase + 15 in
// shared memory, two 8-entry segments; once the pointer leaves the first segment, the
// window slides by one segment and the segment after it is fetched with cp.async (it lands
// while the round's barriers pass).  A pointer that runs past the window reads 8 G entries
// at a time with G independent 16-byte loads (a round takes as long as its longest walk, so
// the round trips to memory count).  lv indexes the vertex's own state.
template <int G>
__device__ __forceinline__ int walk_list(const unsigned short *__restrict__ row, int lv, uint4 *win, unsigned short *ptr,
                                         unsigned short *wbase, const unsigned short *slen, const unsigned char *ms)
{
  int p = ptr[lv], wb = wbase[lv];
  const int L = slen[lv];
  int found = -1;
  while (p < L && found < 0) {
    if (p < wb + 16) {
      const int sg = (p - wb) >> 3;
      const uint4 q4 = win[2 * lv + sg];
      const unsigned w4[4] = { q4.x, q4.y, q4.z, q4.w };
      const int a = wb + 8 * sg;
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int idx = a + e;
        const int u = (int)((w4[e >> 1] >> ((e & 1) * 16)) & 0xFFFFu);
        if (found < 0 && idx >= p && idx < L && !ms[u]) { found = u; p = idx; }
      }
      if (found < 0) p = a + 8;
      continue;
    }
    // past the window: fetch the next 8 G entries with G independent loads
    const int a = p & ~7;
    uint4 g4[G];
#pragma unroll
    for (int j = 0; j < G; ++j)
      if (a + 8 * j < L) g4[j] = *(const uint4 *)(row + a + 8 * j);
#pragma unroll
    for (int j = 0; j < G; ++j) {
      if (found >= 0 || a + 8 * j >= L) continue;
      const unsigned w4[4] = { g4[j].x, g4[j].y, g4[j].z, g4[j].w };
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int idx = a + 8 * j + e;
        const int u = (int)((w4[e >> 1] >> ((e & 1) * 16)) & 0xFFFFu);
        if (found < 0 && idx >= p && idx < L && !ms[u]) { found = u; p = idx; }
      }
      if (found >= 0) {
        // the window restarts at the segment of the find
        wb = a + 8 * j;
        win[2 * lv] = g4[j];
        if (j < G - 1 && wb + 8 < L) win[2 * lv + 1] = g4[j + 1];
        else if (wb + 8 < L) cp_async16(&win[2 * lv + 1], row + wb + 8);
      }
    }
    if (found < 0) p = a + 8 * G;
  }
  if (found < 0) p = L;
  else if (p >= wb + 8 && p < wb + 16) {
    // the first segment is used up: slide the window and fetch the segment after it
    win[2 * lv] = win[2 * lv + 1];
    wb += 8;
    if (wb + 8 < L) cp_async16(&win[2 * lv + 1], row + wb + 8);
  }
  cp_async_commit();
  ptr[lv] = (unsigned short)p;
  wbase[lv] = (unsigned short)wb;
  return found;
}

// a vertex's list state at the start of the matching
__device__ __forceinline__ void walk_init(const unsigned short *__restrict__ row, int L, int lv, uint4 *win, unsigned short *ptr,
                                          unsigned short *wbase, unsigned short *slen)
{
  ptr[lv] = 0;
  wbase[lv] = 0;
  slen[lv] = (unsigned short)L;
  win[2 * lv] = ((const uint4 *)row)[0];
  if (L > 8) win[2 * lv + 1] = ((const uint4 *)row)[1];
}

// By one block, after the matching: the matched pairs ranked by (weight key, tie key),
// descending; the first N_2 are this step's pivots (the STEP array, rank order); the
// columns outside them; the step's scalars.  ms is free scratch here.
template <typename T>
__device__ void select_finish(State *st, const double *__restrict__ Wm, int n, int n_2, int np, int rounds,
                              const int2 *pairs, unsigned long long *skey, unsigned *stie, int *sidx, unsigned char *ms,
                              Piv<T> *piv, int *unp, Trace &tr, int *s_nunp)
{
  const int tid = threadIdx.x, nth = blockDim.x;
  const int s2 = pow2ceil(n / 2 > 0 ? n / 2 : 1);
  for (int i = tid; i < s2; i += nth) {
    if (i < np) {
      const int2 pr = pairs[i];
      skey[i] = wkey(Wm[(long long)pr.x * n + pr.y]);
      stie[i] = tkey(pr.x, pr.y);
      sidx[i] = i;
    }
    else { skey[i] = 0ULL; stie[i] = 0u; sidx[i] = -1; }
  }
  __syncthreads();
  bitonic_desc(skey, stie, sidx, s2);
  const int sl = (np < n_2) ? np : n_2;
  for (int v = tid; v < n; v += nth) ms[v] = 0;
  __syncthreads();
  for (int r = tid; r < sl; r += nth) {
    const int2 pr = pairs[sidx[r]];
    ms[pr.x] = 1;
    ms[pr.y] = 1;
    Piv<T> &pv = piv[r];
    pv.p = pr.x;
    pv.q = pr.y;
    pv.w = Wm[(long long)pr.x * n + pr.y];
  }
  __syncthreads();
  for (int v = tid; v < n; v += nth)
    if (!ms[v]) unp[atomicAdd(s_nunp, 1)] = v;
  __syncthreads();
  if (tid == 0) {
    st->sl = sl;
    st->nl = 0;
    st->err = 0;
    st->nunp = *s_nunp;
    st->rounds = rounds;
    if (sl <= 0) {
      // DSTEP_EXEC returns with SL = 0: the loop ends with INFO = S (src/D/dstep.F90:421, 575-582)
      st->info = st->steps;
      st->stop = 1;
      if (st->trace_on && st->trace_steps < st->trace_cap_steps) {
        const int s = st->trace_steps++;
        tr.sl[s] = 0; tr.nl[s] = -1; tr.tw[s] = -0.0; tr.trig[s] = 0; tr.hyp[s] = 0; tr.rounds[s] = rounds;
      }
    }
    else st->pending = 1;
  }
}

// one block: the end of the previous step, the matching rounds, the ranking of the
// matched pairs and the first N_2 of them (the pivots of this step, rank order),
// and the columns outside the pivot set.
// A round is two barriers: (A) every free vertex finds its best free partner, the first
// free entry of its ranked list from its pointer on (walk_list); (B) mutual proposals
// are matched.
template <typename T>
__global__ void __launch_bounds__(SEL_THREADS, 1)
k_select(State *st, const double *__restrict__ Wm, const int *__restrict__ J, int n, int n_2,
         const unsigned short *__restrict__ list, const int *__restrict__ len, Piv<T> *piv, int *unp, Trace tr)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int s2 = pow2ceil(n / 2 > 0 ? n / 2 : 1);
  unsigned long long *skey = (unsigned long long *)smem_raw;  // [s2]
  unsigned *stie = (unsigned *)(skey + s2);                   // [s2]
  int *sidx = (int *)(stie + s2);                             // [s2]
  int2 *pairs = (int2 *)(sidx + s2);                          // [n/2 + 1]
  uint4 *win = (uint4 *)(pairs + (n / 2 + 1) + ((n / 2 + 1) & 1)); // [n][2]: list entries wbase .. wbase + 15
  int *best = (int *)(win + 2 * n);                           // [n]
  unsigned short *ptr = (unsigned short *)(best + n);         // [n]
  unsigned short *wbase = ptr + n;                            // [n]
  unsigned short *slen = wbase + n;                           // [n]
  unsigned char *ms = (unsigned char *)(slen + n);            // [n]: 0 free, 1 matched, 2 retired
  __shared__ int s_stop, s_cnt, s_nunp, s_rounds;

  const int tid = threadIdx.x, nth = blockDim.x, ld = list_ld(n);
  if (tid == 0) {
    end_of_step<T>(st, piv, J, tr);
    s_stop = st->stop;
    s_cnt = 0; s_nunp = 0; s_rounds = 0;
  }
  __syncthreads();
  if (s_stop) return;
  for (int v = tid; v < n; v += nth) {
    ms[v] = 0;
    walk_init(list + (long long)v * ld, len[v], v, win, ptr, wbase, slen);
  }
  __syncthreads();

  for (int round = 0; round <= n / 2 + 1; ++round) {
    cp_async_wait<0>();  // this thread's window refills of the last round
    // phase A: the best free partner of every free vertex
    for (int v = tid; v < n; v += nth)
      if (!ms[v]) best[v] = walk_list<4>(list + (long long)v * ld, v, win, ptr, wbase, slen, ms);
    __syncthreads();
    // phase B: mutual proposals are matched; a vertex without a candidate retires
    int got = 0;
    for (int v = tid; v < n; v += nth) {
      if (ms[v]) continue;
      const int u = best[v];
      if (u < 0) { ms[v] = 2; continue; }
      if (v < u && best[u] == v) {
        ms[v] = 1;
        ms[u] = 1;
        pairs[atomicAdd(&s_cnt, 1)] = make_int2(v, u);
        got = 1;
      }
    }
    if (tid == 0) s_rounds = round + 1;
    if (!__syncthreads_or(got)) break;
  }
  cp_async_wait<0>();
  select_finish<T>(st, Wm, n, n_2, s_cnt, s_rounds, pairs, skey, stie, sidx, ms, piv, unp, tr, &s_nunp);
}

// The same matching by a cluster of SEL_CLUSTER blocks sharing its state through
// distributed shared memory (plain loads, stores and atomics; no multicast).  Block c owns
// the vertices v = c (mod SEL_CLUSTER) and their list windows; every block keeps a replica
// of every vertex's state (free, matched, retired), which phase B updates in all blocks.
// A round: (A) every block walks its own free vertices' lists; cluster barrier; (B) a free
// vertex whose best partner u proposes back (u's block holds best[u]) is matched with it,
// the pair goes to block 0's list and both states change in every replica; cluster
// barrier; every block reads the round's match count from block 0 and stops when it is 0.
// Block 0 then ranks the matched pairs as the one-block kernel does.
#define SEL_CLUSTER 8
#define SEL_CTHREADS 256

size_t select_cluster_smem(int n)
{
  const int s2 = pow2ceil(n / 2 > 0 ? n / 2 : 1);
  const int np = (n / 2 + 1) + ((n / 2 + 1) & 1);
  const int nl = (n + SEL_CLUSTER - 1) / SEL_CLUSTER;
  return (size_t)s2 * (8 + 4 + 4) + (size_t)np * 8 + (size_t)nl * (32 + 4 + 2 + 2 + 2) + (size_t)n + 16;
}

template <typename T>
__global__ void __cluster_dims__(SEL_CLUSTER, 1, 1) __launch_bounds__(SEL_CTHREADS, 1)
k_select_cluster(State *st, const double *__restrict__ Wm, const int *__restrict__ J, int n, int n_2,
                 const unsigned short *__restrict__ list, const int *__restrict__ len, Piv<T> *piv, int *unp, Trace tr)
{
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int s2 = pow2ceil(n / 2 > 0 ? n / 2 : 1);
  const int nl = (n + SEL_CLUSTER - 1) / SEL_CLUSTER;
  unsigned long long *skey = (unsigned long long *)smem_raw;  // [s2]  (block 0)
  unsigned *stie = (unsigned *)(skey + s2);                   // [s2]  (block 0)
  int *sidx = (int *)(stie + s2);                             // [s2]  (block 0)
  int2 *pairs = (int2 *)(sidx + s2);                          // [n/2 + 1]  (block 0)
  uint4 *win = (uint4 *)(pairs + (n / 2 + 1) + ((n / 2 + 1) & 1)); // [nl][2]: own vertices' windows
  int *best = (int *)(win + 2 * nl);                          // [nl]
  unsigned short *ptr = (unsigned short *)(best + nl);        // [nl]
  unsigned short *wbase = ptr + nl;                           // [nl]
  unsigned short *slen = wbase + nl;                          // [nl]
  unsigned char *ms = (unsigned char *)(slen + nl);           // [n]: replica of every vertex's state
  __shared__ int s_stop, s_cnt, s_nunp, s_rounds, s_got[2];

  const int tid = threadIdx.x, nth = blockDim.x, ld = list_ld(n);
  const int c = (int)cluster.block_rank();
  if (c == 0 && tid == 0) {
    end_of_step<T>(st, piv, J, tr);
    s_stop = st->stop;
    s_cnt = 0; s_nunp = 0; s_rounds = 0; s_got[0] = 0; s_got[1] = 0;
  }
  for (int v = tid; v < n; v += nth) ms[v] = 0;
  for (int lv = tid; lv * SEL_CLUSTER + c < n; lv += nth) {
    const int v = lv * SEL_CLUSTER + c;
    walk_init(list + (long long)v * ld, len[v], lv, win, ptr, wbase, slen);
  }
  int *got0 = cluster.map_shared_rank(s_got, 0);
  int *cnt0 = cluster.map_shared_rank(&s_cnt, 0);
  int2 *pairs0 = cluster.map_shared_rank(pairs, 0);
  cluster.sync();
  const int stop = *cluster.map_shared_rank(&s_stop, 0);
  cluster.sync();  // every block has read block 0's flag
  if (stop) return;

  int rounds = 0;
  for (int round = 0; round <= n / 2 + 1; ++round) {
    cp_async_wait<0>();
    // phase A: the best free partner of each own free vertex
    for (int lv = tid; lv * SEL_CLUSTER + c < n; lv += nth) {
      const int v = lv * SEL_CLUSTER + c;
      if (!ms[v]) best[lv] = walk_list<16>(list + (long long)v * ld, lv, win, ptr, wbase, slen, ms);
    }
    cluster.sync();
    // the next round's match count starts at zero (every block read it two barriers ago)
    if (c == 0 && tid == 0) s_got[(round + 1) & 1] = 0;
    // phase B: mutual proposals are matched; a vertex without a candidate retires
    int got = 0;
    for (int lv = tid; lv * SEL_CLUSTER + c < n; lv += nth) {
      const int v = lv * SEL_CLUSTER + c;
      if (ms[v]) continue;
      const int u = best[lv];
      if (u < 0) {
        for (int b = 0; b < SEL_CLUSTER; ++b) *cluster.map_shared_rank(&ms[v], b) = 2;
        continue;
      }
      if (v < u && *cluster.map_shared_rank(&best[u / SEL_CLUSTER], u % SEL_CLUSTER) == v) {
        for (int b = 0; b < SEL_CLUSTER; ++b) {
          *cluster.map_shared_rank(&ms[v], b) = 1;
          *cluster.map_shared_rank(&ms[u], b) = 1;
        }
        pairs0[atomicAdd(cnt0, 1)] = make_int2(v, u);
        got += 1;
      }
    }
    if (got) atomicAdd(&got0[round & 1], got);
    cluster.sync();
    rounds = round + 1;
    if (!got0[round & 1]) {
      cluster.sync();  // every block has read the count before block 0 goes on alone
      break;
    }
  }
  cp_async_wait<0>();
  if (c != 0) return;  // no block reads another's shared memory after the last barrier
  select_finish<T>(st, Wm, n, n_2, s_cnt, rounds, pairs, skey, stie, sidx, ms, piv, unp, tr, &s_nunp);
}

// per pivot: the 2x2 HSVD of DSTEP_TRANSF's first loop (src/D/dstep.F90:301-326),
// INFO, NL (src/D/dstep.F90:337) and the BA coefficients every rotating block reads
template <typename T>
__global__ void k_pivots(State *st, const T *__restrict__ A, const int *__restrict__ J, int n, Piv<T> *piv, RowRot<T> *rr, int quirk)
{
  if (st->stop) return;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= st->sl) return;
  Piv<T> &pv = piv[r];
  const int p = pv.p, q = pv.q;
  T B[4] = { A[(long long)p * n + p], A[(long long)p * n + q], A[(long long)q * n + p], A[(long long)q * n + q] };
  T V[4], W[4];
  int info = 0;
  Tr<T>::hsvd2(B, J[p], J[q], V, W, JK_TH1FIX, info);
  pv.info = info;
  RowRot<T> x;
  x.p = p; x.q = q; x.flags = 0;
  if (info >= 0) {
#pragma unroll
    for (int k = 0; k < 4; ++k) { pv.V[k] = V[k]; pv.W[k] = W[k]; }
    pv.d[0] = Tr<T>::re(B[M11]);
    pv.d[1] = Tr<T>::re(B[M22]);
    if (info & 2) {
      const typename Tr<T>::R t = Tr<T>::ba(V, quirk);
      x.flags = (t.c1 ? 1 : 0) | (t.c2 ? 2 : 0) | 4;
      x.r1 = t.r1; x.r2 = t.r2; x.m1 = t.m1; x.m2 = t.m2;
    }
    if ((info & 1) && (info & 6)) atomicAdd(&st->nl, 1);
  }
  else
    atomicMin(&st->err, info);
  rr[r] = x;
}

// ---------------------------------------------------------------------------
// ID_NCP = 3: AW_NCP3 (src/shared/atypes.F90:488-592), the best of the greedy walks
// that start at every position of the sorted record list.  For every start offset
// I = 1..IT, AW_NCP2 walks the records I..IT and takes every record whose P and Q
// are both unused, up to N_2; the walk's value is (sum of its weights up to its last
// positive one, added from that one back to the first) + (the sum of the rest, in
// order).  The walk with the largest value wins, ties to the smaller start.  The
// work grows as IT^2, so this strategy is limited to small orders (kNcp3MaxN).
//   k_ncp3_keys    one record per pair: the order key (weight, band, p), NaN last
//   k_ncp3_rank    every record's position by counting the records ahead of it
//   k_ncp3_walks   one warp per start offset: the walk, its length and value
//   k_ncp3_pick    one block: the end of the previous step, the best walk again as
//                  this step's pivots, the columns outside them
// ---------------------------------------------------------------------------
__device__ __forceinline__ int ncp3_tri(int p, int q) { return (q * (q - 1)) / 2 + p; }

__global__ void k_ncp3_keys(const State *st, const double *__restrict__ Wm, int n, unsigned long long *key, unsigned *tie,
                            int *it)
{
  if (st->stop) return;
  const int p = blockIdx.x * 32 + threadIdx.x, q = blockIdx.y * 8 + threadIdx.y;
  if (p >= n || q >= n || p >= q) return;
  const int k = ncp3_tri(p, q);
  const unsigned long long kk = wkey(Wm[(long long)q * n + p]);
  key[k] = kk;
  tie[k] = tkey(p, q);
  if (kk) atomicAdd(it, 1);
}

__global__ void k_ncp3_rank(const State *st, const unsigned long long *__restrict__ key, const unsigned *__restrict__ tie,
                            int nn, int *sorted)
{
  if (st->stop) return;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nn) return;
  const unsigned long long kr = key[r];
  const unsigned tr = tie[r];
  int rank = 0;
  for (int o = 0; o < nn; ++o) rank += kbetter(key[o], tie[o], kr, tr) ? 1 : 0;
  sorted[rank] = r;
}

// the walk from start offset i (0-based) by one warp: picks (p, q) in order into
// pk/qk (when not NULL) and their weights into wv; returns the number of picks
__device__ int ncp3_walk(int i, int it, int n, int n_2, const int *__restrict__ sorted, const unsigned *__restrict__ tie,
                         const double *__restrict__ Wm, unsigned *used, double *wv, int *pk, int *qk)
{
  const int lane = threadIdx.x & 31;
  for (int k = lane; k < (n + 31) / 32; k += 32) used[k] = 0u;
  __syncwarp();
  int picks = 0;
  for (int base = i; base < it && picks < n_2; base += 32) {
    const int idx = base + lane;
    int p = -1, q = -1;
    bool valid = false;
    if (idx < it) {
      const unsigned t = tie[sorted[idx]];
      p = (int)(t & 0xFFFFu);
      q = p + (int)(t >> 16);
      valid = !((used[p >> 5] >> (p & 31)) & 1u) && !((used[q >> 5] >> (q & 31)) & 1u);
    }
    unsigned cand = __ballot_sync(0xFFFFFFFFu, valid);
    while (cand && picks < n_2) {
      const int k = __ffs(cand) - 1;
      const int p1 = __shfl_sync(0xFFFFFFFFu, p, k), q1 = __shfl_sync(0xFFFFFFFFu, q, k);
      if (lane == 0) {
        used[p1 >> 5] |= 1u << (p1 & 31);
        used[q1 >> 5] |= 1u << (q1 & 31);
        wv[picks] = Wm[(long long)q1 * n + p1];
        if (pk) { pk[picks] = p1; qk[picks] = q1; }
      }
      ++picks;
      valid = valid && (lane > k) && p != p1 && p != q1 && q != p1 && q != q1;
      cand = __ballot_sync(0xFFFFFFFFu, valid);
    }
    __syncwarp();
  }
  __syncwarp();
  return picks;
}

// the value of a walk (AW_NCP3's MYWP + MYWN)
__device__ double ncp3_value(const double *wv, int sl)
{
  int l = 0;
  for (int k = sl; k >= 1; --k)
    if (wv[k - 1] > 0.0) { l = k; break; }
  double wp = 0.0, wn = 0.0;
  for (int k = l; k >= 1; --k) wp = __dadd_rn(wp, wv[k - 1]);
  for (int k = l + 1; k <= sl; ++k) wn = __dadd_rn(wn, wv[k - 1]);
  return __dadd_rn(wp, wn);
}

#define NCP3_WARPS 8

__global__ void __launch_bounds__(NCP3_WARPS * 32)
k_ncp3_walks(const State *st, const int *__restrict__ itp, const int *__restrict__ sorted, const unsigned *__restrict__ tie,
             const double *__restrict__ Wm, int n, int n_2, double *val, int *len)
{
  if (st->stop) return;
  __shared__ unsigned used[NCP3_WARPS][kNcp3MaxN / 32];
  __shared__ double wv[NCP3_WARPS][kNcp3MaxN / 2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * NCP3_WARPS + warp, it = *itp;
  if (i >= it) return;
  const int sl = ncp3_walk(i, it, n, n_2, sorted, tie, Wm, used[warp], wv[warp], nullptr, nullptr);
  if (lane == 0) {
    val[i] = ncp3_value(wv[warp], sl);
    len[i] = sl;
  }
}

template <typename T>
__global__ void __launch_bounds__(256)
k_ncp3_pick(State *st, const int *__restrict__ itp, const int *__restrict__ sorted, const unsigned *__restrict__ tie,
            const double *__restrict__ Wm, const int *__restrict__ J, int n, int n_2, const double *__restrict__ val,
            Piv<T> *piv, int *unp, int *itc, Trace tr)
{
  __shared__ int s_stop, s_best, s_sl, s_nunp;
  __shared__ double bv[256];
  __shared__ int bi[256];
  __shared__ unsigned used[kNcp3MaxN / 32];
  __shared__ double wv[kNcp3MaxN / 2];
  __shared__ int pk[kNcp3MaxN / 2], qk[kNcp3MaxN / 2];
  __shared__ unsigned char ms[kNcp3MaxN];
  const int tid = threadIdx.x;
  if (tid == 0) {
    end_of_step<T>(st, piv, J, tr);
    s_stop = st->stop;
    s_nunp = 0;
  }
  __syncthreads();
  const int it = *itp;
  if (s_stop) {
    if (tid == 0) *itc = 0;
    return;
  }
  // the best walk: the largest value, ties to the smaller start
  double b = 0.0;
  int bj = -1;
  for (int i = tid; i < it; i += blockDim.x) {
    const double v = val[i];
    if (bj < 0 || !(v <= b)) { b = v; bj = i; }
  }
  bv[tid] = b;
  bi[tid] = bj;
  __syncthreads();
  if (tid == 0) {
    double bb = 0.0;
    int bb_i = -1;
    for (int t = 0; t < (int)blockDim.x; ++t) {
      if (bi[t] < 0) continue;
      if (bb_i < 0 || !(bv[t] <= bb) || (bv[t] == bb && bi[t] < bb_i)) { bb = bv[t]; bb_i = bi[t]; }
    }
    s_best = bb_i;
  }
  __syncthreads();
  if (tid < 32) {
    const int sl = (s_best >= 0) ? ncp3_walk(s_best, it, n, n_2, sorted, tie, Wm, used, wv, pk, qk) : 0;
    if (tid == 0) s_sl = sl;
  }
  for (int v = tid; v < n; v += blockDim.x) ms[v] = 0;
  __syncthreads();
  const int sl = s_sl;
  for (int r = tid; r < sl; r += blockDim.x) {
    ms[pk[r]] = 1;
    ms[qk[r]] = 1;
    Piv<T> &pv = piv[r];
    pv.p = pk[r];
    pv.q = qk[r];
    pv.w = wv[r];
  }
  __syncthreads();
  for (int v = tid; v < n; v += blockDim.x)
    if (!ms[v]) unp[atomicAdd(&s_nunp, 1)] = v;
  __syncthreads();
  if (tid == 0) {
    *itc = 0;  // the record count of the next step starts from zero
    st->sl = sl;
    st->nl = 0;
    st->err = 0;
    st->nunp = s_nunp;
    st->rounds = it;
    if (sl <= 0) {
      st->info = st->steps;
      st->stop = 1;
      if (st->trace_on && st->trace_steps < st->trace_cap_steps) {
        const int s = st->trace_steps++;
        tr.sl[s] = 0; tr.nl[s] = -1; tr.tw[s] = -0.0; tr.trig[s] = 0; tr.hyp[s] = 0; tr.rounds[s] = it;
      }
    }
    else st->pending = 1;
  }
}

size_t select_smem(int n)
{
  const int s2 = pow2ceil(n / 2 > 0 ? n / 2 : 1);
  const int np = (n / 2 + 1) + ((n / 2 + 1) & 1);
  return (size_t)s2 * (8 + 4 + 4) + (size_t)np * 8 + (size_t)n * (32 + 4 + 2 + 2 + 2 + 1) + 16;
}

// k_colsort instantiations: records per thread E = pow2ceil(n) / SORT_THREADS
int colsort_e(int n)
{
  const int s2 = pow2ceil(n);
  return s2 <= SORT_THREADS ? 1 : s2 / SORT_THREADS;
}
// ---------------------------------------------------------------------------
// the fused transformations of one step (src/D/dstep.F90:301-346).
// Block b < SL owns pivot b's column pair (p, q); the other blocks own two
// columns outside the pivot set.  Each block: load its columns of A; apply the
// row rotations of all pivots (BA of phase 1); then, for a pivot block and when no
// pivot failed, the column rotation AB (phase 2) and the diagonal write-back; store;
// then rotate the columns p, q of U (by V^T / V^H) and of Z (by W), phase 1.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256)
k_rotate(const State *st, T *__restrict__ A, T *__restrict__ U, T *__restrict__ Z, int n, const Piv<T> *__restrict__ piv,
         const RowRot<T> *__restrict__ rr, const int *__restrict__ unp)
{
  if (st->stop) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *col = (T *)smem_raw;
  const int sl = st->sl, b = blockIdx.x;
  int c0, c1 = -1, k = -1;
  if (b < sl) { k = b; c0 = piv[k].p; c1 = piv[k].q; }
  else {
    const int j = 2 * (b - sl), nu = st->nunp;
    if (j >= nu) return;
    c0 = unp[j];
    if (j + 1 < nu) c1 = unp[j + 1];
  }
  T *A0 = A + (long long)c0 * n, *A1 = (c1 >= 0) ? (A + (long long)c1 * n) : nullptr;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    col[i] = A0[i];
    if (A1) col[n + i] = A1[i];
  }
  __syncthreads();
  // phase 1: rows p_m, q_m of every pivot m (BA)
  for (int m = threadIdx.x; m < sl; m += blockDim.x) {
    const RowRot<T> r = rr[m];
    if (!(r.flags & 4)) continue;
    typename Tr<T>::R t;
    t.c1 = r.flags & 1; t.c2 = (r.flags >> 1) & 1;
    t.r1 = r.r1; t.r2 = r.r2; t.m1 = r.m1; t.m2 = r.m2;
    Tr<T>::apply_ba(t, col[r.p], col[r.q]);
    if (A1) Tr<T>::apply_ba(t, col[n + r.p], col[n + r.q]);
  }
  __syncthreads();
  // phase 2 for the pivot's own column pair, only when no pivot failed
  if (k >= 0 && st->err == 0) {
    const Piv<T> &pv = piv[k];
    const int info = pv.info;
    if (info & 4) {
      T W[4] = { pv.W[0], pv.W[1], pv.W[2], pv.W[3] };
      const typename Tr<T>::R t = Tr<T>::ab(W);
      for (int i = threadIdx.x; i < n; i += blockDim.x) Tr<T>::apply_ab(t, col[i], col[n + i]);
    }
    __syncthreads();
    if (!(info & 8) && threadIdx.x == 0) {
      T d0 = Tr<T>::zero(), d1 = Tr<T>::zero();
      if constexpr (sizeof(T) == sizeof(double)) { *(double *)&d0 = pv.d[0]; *(double *)&d1 = pv.d[1]; }
      else { ((double2 *)&d0)->x = pv.d[0]; ((double2 *)&d1)->x = pv.d[1]; }
      col[c0] = d0;                   // A(p,p)
      col[c1] = Tr<T>::zero();        // A(q,p)
      col[n + c0] = Tr<T>::zero();    // A(p,q)
      col[n + c1] = d1;               // A(q,q)
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    A0[i] = col[i];
    if (A1) A1[i] = col[n + i];
  }
  if (k < 0) return;
  const Piv<T> &pv = piv[k];
  const int info = pv.info;
  if (info < 0) return;
  if (info & 2) {
    T V[4] = { pv.V[0], pv.V[1], pv.V[2], pv.V[3] };
    Tr<T>::ut2(V);
    const typename Tr<T>::R t = Tr<T>::ab(V);
    T *u0 = U + (long long)c0 * n, *u1 = U + (long long)c1 * n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      T x = u0[i], y = u1[i];
      Tr<T>::apply_ab(t, x, y);
      u0[i] = x; u1[i] = y;
    }
  }
  if (info & 4) {
    T W[4] = { pv.W[0], pv.W[1], pv.W[2], pv.W[3] };
    const typename Tr<T>::R t = Tr<T>::ab(W);
    T *z0 = Z + (long long)c0 * n, *z1 = Z + (long long)c1 * n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      T x = z0[i], y = z1[i];
      Tr<T>::apply_ab(t, x, y);
      z0[i] = x; z1[i] = y;
    }
  }
}

// ---------------------------------------------------------------------------
// a batch of independent 2x2 HSVDs (the dtest / ztest kernel, src/D/dtest.F90:35)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_hsvd2_batch(int count, T *A, const int *J, T *U, T *Z, int *info, double th1)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  T a[4], u[4], z[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) a[k] = A[4 * i + k];
  int inf = 0;
  Tr<T>::hsvd2(a, J[2 * i], J[2 * i + 1], u, z, th1, inf);
#pragma unroll
  for (int k = 0; k < 4; ++k) { A[4 * i + k] = a[k]; U[4 * i + k] = u[k]; Z[4 * i + k] = z[k]; }
  info[i] = inf;
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
static int grid1(long long work, int threads)
{
  long long g = (work + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > 148LL * 64) g = 148LL * 64;
  return (int)g;
}

cudaError_t prepare_kernels(int n)
{
  // dynamic shared memory beyond the default 48 KB: two columns of A per k_rotate
  // block, the ranking and matching state of k_select
  cudaError_t e = cudaFuncSetAttribute(k_rotate<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * n * 8);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_hyp_pm, cudaFuncAttributeMaxDynamicSharedMemorySize, SCAN_STAGES * (2 * TW) * SCAN_RS * (int)sizeof(double));
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_rotate<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * n * 16);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_hyp_z_pm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kZSmem);
  const int ss = (int)select_smem(n);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_select<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, ss);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_select<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, ss);
  const int cs = (int)select_cluster_smem(n);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_select_cluster<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, cs);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_select_cluster<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, cs);
  return e;
}

template <typename T>
static cudaError_t init_t(Workspace &w, T *U, T *Z, int learned, int stall_k, int steps0, int fresh, cudaStream_t s)
{
  k_state_init<<<1, 1, 0, s>>>(w.st, learned, stall_k, steps0);
  if (fresh) k_identity2<T><<<grid1((long long)w.n * w.n, 256), 256, 0, s>>>(U, Z, w.n);
  return cudaGetLastError();
}

// the loop state of a new solve (fresh: U = Z = I) or of a loop that went on for
// steps0 steps (U, Z kept)
cudaError_t launch_init(Workspace &w, void *U, void *Z, int learned, int stall_k, int steps0, int fresh, cudaStream_t s)
{
  return w.cplx ? init_t(w, (double2 *)U, (double2 *)Z, learned, stall_k, steps0, fresh, s)
                : init_t(w, (double *)U, (double *)Z, learned, stall_k, steps0, fresh, s);
}

cudaError_t launch_limit(Workspace &w, long long limit, cudaStream_t s)
{
  k_set_limit<<<1, 1, 0, s>>>(w.st, limit);
  return cudaGetLastError();
}

// undo the end of the loop (k_sigma, k_jztj): the diagonal back from SIGMA, and
// J Z^T J again, which gives back Z (a transposition with sign changes)
template <typename T>
static cudaError_t unfinish_t(Workspace &w, T *A, T *Z, const double *sigma, cudaStream_t s)
{
  const int n = w.n, nt = (n + 31) / 32;
  k_unsigma<T><<<grid1(n, 256), 256, 0, s>>>(A, sigma, n);
  k_jztj<T><<<nt * (nt + 1) / 2, dim3(32, 8), 0, s>>>(Z, w.J, n);
  return cudaGetLastError();
}

cudaError_t launch_unfinish(Workspace &w, void *A, void *Z, const double *sigma, cudaStream_t s)
{
  return w.cplx ? unfinish_t(w, (double2 *)A, (double2 *)Z, sigma, s) : unfinish_t(w, (double *)A, (double *)Z, sigma, s);
}

// the row buffer, which also holds a tile's scan parameters before the rows arrive
static_assert(TW * TW * sizeof(HypPar) <= SCAN_STAGES * (2 * TW) * SCAN_RS * sizeof(double),
              "a tile's scan parameters must fit in the row buffer");

static void hyp_d_launch(Workspace &w, const double *A, cudaStream_t s)
{
  const int nt = ((w.n_plus + TW - 1) / TW) * ((w.n_minus + TW - 1) / TW);
  const size_t smem = SCAN_STAGES * (2 * TW) * SCAN_RS * sizeof(double);
  k_hyp_pm<<<nt, SCAN_THREADS, smem, s>>>(w.st, A, w.plus, w.minus, w.n_plus, w.n_minus, w.n, w.Wm);
}

template <typename T>
static cudaError_t weights_t(Workspace &w, const T *A, cudaStream_t s)
{
  const int n = w.n;
  dim3 bt(32, 8), gt((n + 31) / 32, (n + 7) / 8);
  k_weights_trig<T><<<gt, bt, 0, s>>>(w.st, A, w.J, w.Wm, n);
  if (w.n_plus > 0 && w.n_minus > 0) {
    // the pipelined real kernel once its tiles fill the GPU; 16 x 16 / 8 x 8 tiles otherwise
    if (sizeof(T) == sizeof(double) && (long long)w.n_plus * w.n_minus >= 512LL * 148 * 2) {
      hyp_d_launch(w, (const double *)A, s);
    }
    else if (sizeof(T) == sizeof(double2)) {
      // complex: the magnitudes of all entries once, then the tiles
      const long long nn = (long long)n * n;
      k_absmat<<<(unsigned)((nn + 255) / 256 < 4096 ? (nn + 255) / 256 : 4096), 256, 0, s>>>(w.st, (const double2 *)A, nn,
                                                                                              w.mag);
      if ((long long)w.n_plus * w.n_minus >= (long long)ZTP * ZTM * 148) {
        // the pipelined tiles once they fill the GPU
        const int nt = ((w.n_plus + ZTP - 1) / ZTP) * ((w.n_minus + ZTM - 1) / ZTM);
        k_hyp_z_pm<<<nt, ZTHREADS, kZSmem, s>>>(w.st, (const double2 *)A, w.mag, w.plus, w.minus, w.n_plus, w.n_minus, n,
                                                w.Wm);
      }
      else if ((long long)w.n_plus * w.n_minus >= 256LL * 148 * 4) {
        dim3 gh((w.n_plus + 15) / 16, (w.n_minus + 15) / 16);
        k_weights_hyp_z<16, 16><<<gh, 256, 0, s>>>(w.st, (const double2 *)A, w.mag, w.plus, w.minus, w.n_plus, w.n_minus,
                                                  w.Wm, n);
      }
      else {
        dim3 gh((w.n_plus + 7) / 8, (w.n_minus + 7) / 8);
        k_weights_hyp_z<8, 8><<<gh, 64, 0, s>>>(w.st, (const double2 *)A, w.mag, w.plus, w.minus, w.n_plus, w.n_minus,
                                               w.Wm, n);
      }
    }
    else if ((long long)w.n_plus * w.n_minus >= 256LL * 148 * 4) {
      dim3 gh((w.n_plus + 15) / 16, (w.n_minus + 15) / 16);
      k_weights_hyp<T, 16, 16><<<gh, 256, 0, s>>>(w.st, A, w.plus, w.minus, w.n_plus, w.n_minus, w.Wm, n);
    }
    else {
      dim3 gh((w.n_plus + 7) / 8, (w.n_minus + 7) / 8);
      k_weights_hyp<T, 8, 8><<<gh, 64, 0, s>>>(w.st, A, w.plus, w.minus, w.n_plus, w.n_minus, w.Wm, n);
    }
  }
  return cudaGetLastError();
}

cudaError_t launch_weights(Workspace &w, const void *A, cudaStream_t s)
{
  return w.cplx ? weights_t(w, (const double2 *)A, s) : weights_t(w, (const double *)A, s);
}

static cudaError_t colsort(Workspace &w, cudaStream_t s)
{
  const int n = w.n;
  switch (colsort_e(n)) {
  case 1: k_colsort<1><<<n, SORT_THREADS, 0, s>>>(w.st, w.Wm, n, w.list, w.rank, w.len); break;
  case 2: k_colsort<2><<<n, SORT_THREADS, 0, s>>>(w.st, w.Wm, n, w.list, w.rank, w.len); break;
  case 4: k_colsort<4><<<n, SORT_THREADS, 0, s>>>(w.st, w.Wm, n, w.list, w.rank, w.len); break;
  case 8: k_colsort<8><<<n, SORT_THREADS, 0, s>>>(w.st, w.Wm, n, w.list, w.rank, w.len); break;
  case 16: k_colsort<16><<<n, SORT_THREADS, 0, s>>>(w.st, w.Wm, n, w.list, w.rank, w.len); break;
  default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <typename T>
static cudaError_t select_t(Workspace &w, const T *A, int n_2, cudaStream_t s)
{
  const int n = w.n;
  cudaError_t e = cudaSuccess;
  if (w.id_ncp == 3) {
    // AW_NCP3: every start offset's walk, then the best one
    const int nn = n * (n - 1) / 2;
    k_ncp3_keys<<<dim3((n + 31) / 32, (n + 7) / 8), dim3(32, 8), 0, s>>>(w.st, w.Wm, n, w.n3key, w.n3tie, w.n3it);
    k_ncp3_rank<<<(nn + 255) / 256, 256, 0, s>>>(w.st, w.n3key, w.n3tie, nn, w.n3sorted);
    k_ncp3_walks<<<(nn + NCP3_WARPS - 1) / NCP3_WARPS, NCP3_WARPS * 32, 0, s>>>(w.st, w.n3it, w.n3sorted, w.n3tie, w.Wm, n,
                                                                                 n_2, w.n3val, w.n3len);
    k_ncp3_pick<T><<<1, 256, 0, s>>>(w.st, w.n3it, w.n3sorted, w.n3tie, w.Wm, w.J, n, n_2, w.n3val, (Piv<T> *)w.piv, w.unp,
                                     w.n3it, w.tr);
  }
  else {
    e = colsort(w, s);
    if (e != cudaSuccess) return e;
    if (n >= kSelClusterMinN)
      k_select_cluster<T><<<SEL_CLUSTER, SEL_CTHREADS, select_cluster_smem(n), s>>>(w.st, w.Wm, w.J, n, n_2, w.list, w.len,
                                                                                  (Piv<T> *)w.piv, w.unp, w.tr);
    else
      k_select<T><<<1, SEL_THREADS, select_smem(n), s>>>(w.st, w.Wm, w.J, n, n_2, w.list, w.len, (Piv<T> *)w.piv, w.unp,
                                                       w.tr);
  }
  if (A) {
    const int half = n / 2 > 0 ? n / 2 : 1;
    k_pivots<T><<<(half + 127) / 128, 128, 0, s>>>(w.st, A, w.J, n, (Piv<T> *)w.piv, (RowRot<T> *)w.rowrot, w.zba_quirk);
  }
  return cudaGetLastError();
}

cudaError_t launch_match(Workspace &w, int n_2, cudaStream_t s)
{
  return select_t<double>(w, (const double *)nullptr, n_2, s);
}

template <typename T>
static cudaError_t step_t(Workspace &w, T *A, T *U, T *Z, int n_2, cudaStream_t s)
{
  const int n = w.n;
  cudaError_t e = weights_t(w, (const T *)A, s);
  if (e != cudaSuccess) return e;
  // a learned solve: the scorer ranks the scanned hyperbolic pairs (the exact scan kernels
  // above return at once in its learned steps)
  if (w.learned && (e = launch_learned_weights(w, A, s)) != cudaSuccess) return e;
  e = select_t(w, (const T *)A, n_2, s);
  if (e != cudaSuccess) return e;
  k_rotate<T><<<(n + 1) / 2, 256, 2 * (size_t)n * sizeof(T), s>>>(w.st, A, U, Z, n, (const Piv<T> *)w.piv,
                                                                 (const RowRot<T> *)w.rowrot, w.unp);
  if (w.learned && (e = cudaGetLastError()) == cudaSuccess) e = launch_offnorm(w, A, s);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

cudaError_t launch_step(Workspace &w, void *A, void *U, void *Z, int n_2, cudaStream_t s)
{
  return w.cplx ? step_t(w, (double2 *)A, (double2 *)U, (double2 *)Z, n_2, s)
                : step_t(w, (double *)A, (double *)U, (double *)Z, n_2, s);
}

template <typename T>
static cudaError_t finish_t(Workspace &w, T *A, T *Z, double *sigma, cudaStream_t s)
{
  const int n = w.n, nt = (n + 31) / 32;
  k_sigma<T><<<grid1(n, 256), 256, 0, s>>>(A, sigma, n);
  k_jztj<T><<<nt * (nt + 1) / 2, dim3(32, 8), 0, s>>>(Z, w.J, n);
  return cudaGetLastError();
}

cudaError_t launch_finish(Workspace &w, void *A, void *Z, double *sigma, cudaStream_t s)
{
  return w.cplx ? finish_t(w, (double2 *)A, (double2 *)Z, sigma, s) : finish_t(w, (double *)A, (double *)Z, sigma, s);
}

// FP64 FMA throughput probe: 8 independent dependent chains per thread
__global__ void k_fp64_peak(double *out, int reps)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double x0 = 1.0 + t * 1e-12, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  const double b = 0.999999, c = 1e-9;
  for (int r = 0; r < reps; ++r) {
    x0 = fma(x0, b, c); x1 = fma(x1, b, c); x2 = fma(x2, b, c); x3 = fma(x3, b, c);
    x4 = fma(x4, b, c); x5 = fma(x5, b, c); x6 = fma(x6, b, c); x7 = fma(x7, b, c);
  }
  out[t] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}

double fp64_peak()
{
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = nsm * 16, threads = 256, reps = 4000;
  double *out = nullptr;
  if (cudaMalloc(&out, (size_t)blocks * threads * sizeof(double)) != cudaSuccess) { cudaGetLastError(); return -1.0; }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_fp64_peak<<<blocks, threads>>>(out, 100);
  float best = 1e30f;
  for (int it = 0; it < 3; ++it) {
    cudaEventRecord(e0);
    k_fp64_peak<<<blocks, threads>>>(out, reps);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (cudaGetLastError() != cudaSuccess) return -1.0;
  return 2.0 * 8.0 * reps * (double)blocks * threads / (best * 1e-3) / 1e12;
}

cudaError_t launch_hsvd2_batch(int cplx, int count, void *A, const int *J, void *U, void *Z, int *info, double th1, cudaStream_t s)
{
  if (count <= 0) return cudaSuccess;
  if (cplx) k_hsvd2_batch<double2><<<(count + 127) / 128, 128, 0, s>>>(count, (double2 *)A, J, (double2 *)U, (double2 *)Z, info, th1);
  else k_hsvd2_batch<double><<<(count + 127) / 128, 128, 0, s>>>(count, (double *)A, J, (double *)U, (double *)Z, info, th1);
  return cudaGetLastError();
}


// ---------------------------------------------------------------------------
// Pair weights with no allocation at all (jk_dweights_noalloc).  Some callers may
// not allocate device memory at the point where they need the weights: cudaMalloc
// and cudaFree synchronise the whole device, which stalls a caller's other streams
// inside a latency-bound loop, and they fail outright for a caller whose device
// memory has already been handed to its own pool allocator.  For them the only
// state the two weight kernels need besides A and W (the stop flag, J and the
// "+"/"-" index lists) lives in the file-scope array below, sized for N up to
// kNoallocMaxN.  The pipelined tile kernel needs per-tile parameter storage that
// grows with N^2, so this form always uses the 16 x 16 / 8 x 8 tile kernel, whose
// results are the same bit for bit.
//
// The array is shared by every call on a device: two calls whose kernels overlap
// (different streams with no ordering between them) overwrite each other's J and
// index lists and race.  The State record must start at zero (stop == 0); every
// call copies a zeroed record in together with J and the index lists.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kScratchState = 256;  // State, padded to the alignment of what follows
static_assert(sizeof(State) <= kScratchState, "State does not fit its scratch slot");
constexpr size_t kScratchBytes = kScratchState + 3 * (size_t)kNoallocMaxN * sizeof(int);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void *g_scratch_addr[kMaxDevices];  // device address of g_noalloc_scratch, per device

// Set-up, once per device, with that device current: the device address of the
// array.  The first call on a device therefore makes this runtime call, and should
// come before any stream capture on that device.
cudaError_t scratch_address(int dev, unsigned char **out)
{
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void *a = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&a, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = a;
  }
  *out = (unsigned char *)g_scratch_addr[dev];
  return cudaSuccess;
}

}  // namespace

cudaError_t launch_weights_noalloc(int n, const double *A, const int *J, double *W, cudaStream_t s)
{
  if (n < 1 || n > kNoallocMaxN) return cudaErrorInvalidValue;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  unsigned char *d = nullptr;
  if ((e = scratch_address(dev, &d)) != cudaSuccess) return e;
  // the image of the scratch on the host stack: a zeroed State, J, then the indices
  // with J = +1 and with J = -1 in ascending order
  alignas(16) unsigned char h[kScratchBytes];
  memset(h, 0, kScratchState);
  int *hj = (int *)(h + kScratchState), *hp = hj + kNoallocMaxN, *hm = hp + kNoallocMaxN;
  int np = 0, nm = 0;
  for (int i = 0; i < n; ++i) {
    hj[i] = J[i];
    if (J[i] == 1) hp[np++] = i;
    else hm[nm++] = i;
  }
  // pageable source: the call returns once the bytes are staged, so the stack image may go
  if ((e = cudaMemcpyAsync(d, h, kScratchBytes, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
  const State *st = (const State *)d;
  const int *dj = (const int *)(d + kScratchState), *dp = dj + kNoallocMaxN, *dm = dp + kNoallocMaxN;
  dim3 bt(32, 8), gt((n + 31) / 32, (n + 7) / 8);
  k_weights_trig<double><<<gt, bt, 0, s>>>(st, A, dj, W, n);
  if (np > 0 && nm > 0) {
    if ((long long)np * nm >= 256LL * 148 * 4) {
      dim3 gh((np + 15) / 16, (nm + 15) / 16);
      k_weights_hyp<double, 16, 16><<<gh, 256, 0, s>>>(st, A, dp, dm, np, nm, W, n);
    }
    else {
      dim3 gh((np + 7) / 8, (nm + 7) / 8);
      k_weights_hyp<double, 8, 8><<<gh, 64, 0, s>>>(st, A, dp, dm, np, nm, W, n);
    }
  }
  return cudaGetLastError();
}

}  // namespace jk
