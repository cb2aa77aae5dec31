// jk_batch.cu -- the batched persistent solver: many independent real matrices of
// small order (N <= 128), each solved by one thread block from the start to the end
// of its step loop (DSTEP_LOOP, src/D/dstep.F90:472-604), all in a single launch.
//
// A block keeps its matrix A in shared memory for the whole solve, with its columns
// permuted so that the J = +1 columns come first (every hyperbolic pair is then a
// (+ column, - column) pair and neighbouring threads read neighbouring columns), the
// pair weights of the current step as a packed upper triangle, and the pivots of the
// step.  U and Z stay in global memory (their columns p, q are touched once per pivot).
// Each step runs, separated by block barriers:
//   weights    DMAGF2T / DMAGF2H (+ ABODNDF2) of every pair, the arithmetic of the
//              single-matrix kernels (src/D/dstep.F90:12-72, 189-219)
//   selection  the greedy non-colliding pivots (AW_SRT* + AW_NCP1/2,
//              src/shared/atypes.F90:85-484) as the greedy matching, by the Suitor
//              method (warp-wide proposals that displace worse suitors, shared-memory
//              compare-and-swap, no barrier per round); matched pairs ranked by the
//              record order, the first N_2 kept
//   pivots     the 2x2 HSVDs (src/D/dstep.F90:301-326), NL and the error minimum
//   rotations  all row rotations (BA) of A and the column rotations of U and Z, then,
//              if no pivot failed, the column rotations (AB) of A and the diagonal
//              write-back (src/D/dstep.F90:301-346)
//   loop test  SL := MIN(SL, NL), S, INFO (src/D/dstep.F90:564-583)
// and at the end SIGMA, the zeroed diagonal and Z := J Z^T J (src/D/dstep.F90:447-468,
// 585-602).  Blocks take matrices from a work counter in the host's order (largest
// first), so the launch is persistent and balances itself.
#include "jk_internal.h"
#include "jk_device.cuh"

namespace jk {

namespace {

struct BPiv {
  Rot ba;          // BA coefficients of V (rows of A), valid when info >= 0 and info & 2
  Rot tu;          // AB coefficients of UT2(V) (columns of U), same validity
  Rot tz;          // AB coefficients of W (columns of A and Z), valid when info & 4
  double d0, d1;   // the new diagonal
  int p, q, info, pad;
};

__host__ __device__ __forceinline__ int tri(int p, int q) { return (q * (q - 1)) / 2 + p; }  // p < q

__host__ __device__ __forceinline__ size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

// shared-memory layout for the largest order nm of the batch
struct BLayout {
  size_t a, w, piv, pairs, rank, pos, vlist, jv, best, ms, cn, total;
  __host__ __device__ explicit BLayout(int nm)
  {
    const int h = nm / 2 + 1;
    a = 0;
    w = align16(a + (size_t)nm * (nm + 1) * sizeof(double));
    piv = align16(w + (size_t)(nm * (nm - 1) / 2 + 1) * sizeof(double));
    pairs = align16(piv + (size_t)h * sizeof(BPiv));
    rank = align16(pairs + (size_t)h * sizeof(int2));
    pos = align16(rank + (size_t)h * sizeof(int));
    vlist = align16(pos + (size_t)nm * sizeof(int));
    jv = align16(vlist + (size_t)nm * sizeof(int));
    best = align16(jv + (size_t)nm * sizeof(int));
    ms = align16(best + (size_t)nm * sizeof(int));
    cn = align16(ms);
    total = cn + (size_t)nm * sizeof(double);
  }
};

// the record order (AW_CMP): larger weight, then larger band q - p, then larger p;
// t = (band << 16) | p
__device__ __forceinline__ bool rbetter(double w1, unsigned t1, double w2, unsigned t2)
{
  return (w1 > w2) || ((w1 == w2) && (t1 > t2));
}

__device__ __forceinline__ unsigned rtie(int p, int q) { return ((unsigned)(q - p) << 16) | (unsigned)p; }

// ABODNDF2's sequential sum over the rows i != p, q of the columns xs (p), ys (q)
// under the AB coefficients t (src/D/dtransf.F90:246-348)
__device__ __forceinline__ void scan_pair(const double *xs, const double *ys, int n, int p, int q, const Rot &t, double &d)
{
  if (t.c1 && t.c2) {
#pragma unroll 4
    for (int i = 0; i < n; ++i) {
      const double x = xs[i], y = ys[i];
      const double xx = __dmul_rn(fma(y, t.r1, x), t.m1);
      const double yy = __dmul_rn(fma(x, t.r2, y), t.m2);
      const double e1 = fma(__dsub_rn(x, xx), __dadd_rn(x, xx), d);
      const double e2 = fma(__dsub_rn(y, yy), __dadd_rn(y, yy), e1);
      d = (i != p && i != q) ? e2 : d;
    }
  }
  else {
    for (int i = 0; i < n; ++i) {
      double x = xs[i], y = ys[i];
      const double x0 = x, y0 = y;
      rot_apply(t, x, y);
      const double e1 = fma(__dsub_rn(x0, x), __dadd_rn(x0, x), d);
      const double e2 = fma(__dsub_rn(y0, y), __dadd_rn(y0, y), e1);
      d = (i != p && i != q) ? e2 : d;
    }
  }
}

// scored: rank the scanned hyperbolic pairs by the Gram form of their weights (squared
// column norms and the column products without rows p, q; one fma per row instead of the
// scan's ten operations), with the fallback rules of the single-matrix scored loop: after
// stall_k steps without a new minimum of the off-norm the next step ranks exactly, a
// scored step without an effective pivot is followed by an exact step (only an exact
// step ends the loop), and once the off-norm exceeds 16 times its minimum the rest of
// the solve ranks exactly
template <int THREADS>
__device__ void solve_one(const BatchItem &it, double *__restrict__ gA, double *__restrict__ gU, double *__restrict__ gZ,
                          const int *__restrict__ gJ, double *__restrict__ gsigma, int *__restrict__ ginfo, int nm,
                          long long cap, int scored, int stall_k, unsigned char *smem)
{
  const BLayout L(nm);
  double *As = (double *)(smem + L.a);
  double *Ws = (double *)(smem + L.w);
  BPiv *pv = (BPiv *)(smem + L.piv);
  int2 *pairs = (int2 *)(smem + L.pairs);
  int *rk = (int *)(smem + L.rank);
  int *pos = (int *)(smem + L.pos);      // vertex -> shared-memory column
  int *vl = (int *)(smem + L.vlist);     // shared-memory column -> vertex (+ columns, then - columns)
  int *Jv = (int *)(smem + L.jv);
  int *suitor = (int *)(smem + L.best);  // per vertex: its current suitor (-1: none)
  double *cn = (double *)(smem + L.cn);  // scored steps: squared off-diagonal column norms
  __shared__ int s_np, s_cnt, s_nl, s_err;
  __shared__ int s_learned, s_lstep, s_retry, s_stall;  // the scored ranking's state
  __shared__ double s_best, s_red[THREADS / 32];

  const int tid = threadIdx.x, n = it.n, lda = n + 1, v_ = tid;
  double *A = gA + it.off, *U = gU + it.off, *Z = gZ + it.off;
  const int *J = gJ + it.joff;

  // J, the column permutation, A into shared memory, U = Z = I
  if (tid < 32) {
    int np = 0;
    for (int b = 0; b < n; b += 32) {
      const int v = b + tid;
      const int jj = (v < n) ? J[v] : 0;
      const unsigned m = __ballot_sync(0xFFFFFFFFu, jj == 1);
      if (v < n) {
        Jv[v] = jj;
        if (jj == 1) pos[v] = np + __popc(m & ((1u << tid) - 1u));
      }
      np += __popc(m);
    }
    int nmn = 0;
    for (int b = 0; b < n; b += 32) {
      const int v = b + tid;
      const bool mi = (v < n) && (J[v] != 1);
      const unsigned m = __ballot_sync(0xFFFFFFFFu, mi);
      if (mi) pos[v] = np + nmn + __popc(m & ((1u << tid) - 1u));
      nmn += __popc(m);
    }
    if (tid == 0) s_np = np;
  }
  __syncthreads();
  for (int v = tid; v < n; v += THREADS) vl[pos[v]] = v;
  for (int k = tid; k < n * n; k += THREADS) {
    const int i = k % n, j = k / n;
    As[pos[j] * lda + i] = A[k];
    const double e = (i == j) ? 1.0 : 0.0;
    U[k] = e;
    Z[k] = e;
  }
  __syncthreads();
  const int np = s_np, nmn = n - np;
  const int nn = n * (n - 1) / 2;
  int steps = 0, info = 0;
  if (tid == 0) {
    s_learned = scored;
    s_lstep = scored;
    s_retry = 0;
    s_stall = 0;
    s_best = __longlong_as_double(0x7FF0000000000000LL);  // +inf
  }
  __syncthreads();

  for (;;) {
    const bool lstep = s_lstep;  // this step ranks by the Gram form
    if (lstep) {
      for (int v = tid; v < n; v += THREADS) {
        const double *c = As + pos[v] * lda;
        double a = 0.0;
        for (int i = 0; i < n; ++i)
          if (i != v) a = fma(c[i], c[i], a);
        cn[v] = a;
      }
      __syncthreads();
    }
    // ---- weights of the trigonometric pairs (DMAGF2T)
    for (int k = tid; k < nn; k += THREADS) {
      int q = (int)((1.0 + sqrt(8.0 * k + 1.0)) * 0.5);
      while (tri(0, q) > k) --q;
      while (tri(0, q + 1) <= k) ++q;
      const int p = k - tri(0, q);
      const int s = Jv[p] + Jv[q];
      if (s != 2 && s != -2) continue;
      const double *cp = As + pos[p] * lda, *cq = As + pos[q] * lda;
      const double app = cp[p], aqp = cp[q], apq = cq[p], aqq = cq[q];
      const bool nz = may_transform(app, aqp, apq, aqq);
      double w;
      if (s == -2) w = (nz || (aqq < app)) ? dasum2(aqp, apq) : nan_w();
      else w = (nz || (app < aqq)) ? dasum2(aqp, apq) : nan_w();
      Ws[k] = w;
    }
    // ---- weights of the hyperbolic pairs (DMAGF2H + ABODNDF2): + column ci, - column cj;
    // with up to 384 threads two pairs per thread, their fma chains interleaved (the
    // 512-thread shape has no registers to spare for it)
    const int nh = np * nmn;
    if (lstep) {
      // the Gram form: per pair the product of its columns without rows p, q
      for (int k = tid; k < nh; k += THREADS) {
        const int ci = k / nmn, cj = np + k % nmn;  // shared-memory columns
        const int a = vl[ci], b = vl[cj];
        const bool a_is_p = a < b;
        const int p = a_is_p ? a : b, q = a_is_p ? b : a;
        const double *xs = As + (a_is_p ? ci : cj) * lda, *ys = As + (a_is_p ? cj : ci) * lda;
        double w, d = 0.0, Z2[4];
        if (hyp_setup_z(xs[p], xs[q], ys[p], ys[q], a_is_p ? 1 : -1, w, d, Z2)) {
          double g = 0.0;
#pragma unroll 4
          for (int i = 0; i < n; ++i) {
            const double e = fma(xs[i], ys[i], g);
            g = (i != p && i != q) ? e : g;
          }
          w = gram_weight(d, Z2, cn[p] - xs[q] * xs[q], cn[q] - ys[p] * ys[p], g);
        }
        if (w < -JK_HUGE) w = nan_w();
        Ws[tri(p, q)] = w;
      }
    }
    else if constexpr (THREADS > 384) {
      for (int k = tid; k < nh; k += THREADS) {
        const int ci = k / nmn, cj = np + k % nmn;  // shared-memory columns
        const int a = vl[ci], b = vl[cj];
        const bool a_is_p = a < b;
        const int p = a_is_p ? a : b, q = a_is_p ? b : a;
        const double *xs = As + (a_is_p ? ci : cj) * lda, *ys = As + (a_is_p ? cj : ci) * lda;
        double w, d = 0.0;
        Rot t;
        if (hyp_setup(xs[p], xs[q], ys[p], ys[q], a_is_p ? 1 : -1, w, d, t)) {
          scan_pair(xs, ys, n, p, q, t, d);
          w = d;
        }
        if (w < -JK_HUGE) w = nan_w();
        Ws[tri(p, q)] = w;
      }
    }
    else
    for (int k0 = tid; k0 < nh; k0 += 2 * THREADS) {
      int pp[2], qq[2];
      const double *xs[2], *ys[2];
      double w[2], d[2];
      Rot t[2];
      bool sc[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int k = k0 + h * THREADS;
        sc[h] = false; w[h] = nan_w(); d[h] = 0.0; pp[h] = 0; qq[h] = 1; xs[h] = As; ys[h] = As;
        if (k < nh) {
          const int ci = k / nmn, cj = np + k % nmn;  // shared-memory columns
          const int a = vl[ci], b = vl[cj];
          const bool a_is_p = a < b;
          pp[h] = a_is_p ? a : b;
          qq[h] = a_is_p ? b : a;
          xs[h] = As + (a_is_p ? ci : cj) * lda;
          ys[h] = As + (a_is_p ? cj : ci) * lda;
          sc[h] = hyp_setup(xs[h][pp[h]], xs[h][qq[h]], ys[h][pp[h]], ys[h][qq[h]], a_is_p ? 1 : -1, w[h], d[h], t[h]);
        }
      }
      if (sc[0] && sc[1] && t[0].c1 && t[0].c2 && t[1].c1 && t[1].c2) {
        // ABODNDF2's sequential sums over the rows i != p, q, two chains at once
#pragma unroll 2
        for (int i = 0; i < n; ++i) {
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const double x = xs[h][i], y = ys[h][i];
            const double xx = __dmul_rn(fma(y, t[h].r1, x), t[h].m1);
            const double yy = __dmul_rn(fma(x, t[h].r2, y), t[h].m2);
            const double e1 = fma(__dsub_rn(x, xx), __dadd_rn(x, xx), d[h]);
            const double e2 = fma(__dsub_rn(y, yy), __dadd_rn(y, yy), e1);
            d[h] = (i != pp[h] && i != qq[h]) ? e2 : d[h];
          }
        }
      }
      else {
#pragma unroll
        for (int h = 0; h < 2; ++h)
          if (sc[h]) scan_pair(xs[h], ys[h], n, pp[h], qq[h], t[h], d[h]);
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (k0 + h * THREADS >= nh) continue;
        double x = sc[h] ? d[h] : w[h];
        if (x < -JK_HUGE) x = nan_w();
        Ws[tri(pp[h], qq[h])] = x;
      }
    }
    for (int v = tid; v < n; v += THREADS) suitor[v] = -1;
    if (tid == 0) { s_cnt = 0; s_nl = 0; s_err = 0; }
    __syncthreads();

    // ---- selection: the greedy matching by the Suitor method (Manne & Halappanavar):
    // a vertex proposes to its best partner whose current suitor offers a worse pair
    // (record order), displacing that suitor, which then proposes in turn.  With a
    // strict total order this ends in the greedy matching, the set of pairs the walk
    // over the sorted records takes, without a barrier per round.  A warp makes one
    // proposal at a time: its lanes scan the partners, a butterfly reduction finds
    // the best open one, lane 0 places it with a compare-and-swap.
    {
      volatile int *vs = suitor;  // other warps change it at any time
      const int lane = tid & 31;
      int guard = 0;
      const int limit = 2 * n * n + 64;
      for (int v0 = tid >> 5; v0 < n && guard <= limit; v0 += THREADS / 32) {
        int cur = v0;
        while (cur >= 0 && guard <= limit) {
          double bw = 0.0;
          unsigned bt = 0u;
          int bu = -1;
          for (int u = lane; u < n; u += 32) {
            if (u == cur) continue;
            const int p = (u < cur) ? u : cur, q = (u < cur) ? cur : u;
            const double w = Ws[tri(p, q)];
            if (w != w) continue;  // NaN: no record
            const unsigned t = rtie(p, q);
            if (bu >= 0 && !rbetter(w, t, bw, bt)) continue;
            const int su = vs[u];
            if (su >= 0) {
              const int p2 = (u < su) ? u : su, q2 = (u < su) ? su : u;
              if (!rbetter(w, t, Ws[tri(p2, q2)], rtie(p2, q2))) continue;
            }
            bw = w; bt = t; bu = u;
          }
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) {
            const double ow = __shfl_xor_sync(0xFFFFFFFFu, bw, off);
            const unsigned ot = __shfl_xor_sync(0xFFFFFFFFu, bt, off);
            const int ou = __shfl_xor_sync(0xFFFFFFFFu, bu, off);
            if (ou >= 0 && (bu < 0 || rbetter(ow, ot, bw, bt))) { bw = ow; bt = ot; bu = ou; }
          }
          if (bu < 0) break;  // no open partner: cur stays unmatched
          int res = -2;
          if (lane == 0) {
            const int s0 = vs[bu];
            bool still = (s0 < 0);
            if (!still) {
              const int p2 = (bu < s0) ? bu : s0, q2 = (bu < s0) ? s0 : bu;
              still = rbetter(bw, bt, Ws[tri(p2, q2)], rtie(p2, q2));
            }
            if (still && atomicCAS(&suitor[bu], s0, cur) == s0) res = s0;
          }
          res = __shfl_sync(0xFFFFFFFFu, res, 0);
          ++guard;
          if (res == -2) continue;  // overtaken meanwhile: look again
          cur = res;                // the displaced suitor proposes next
        }
      }
      if (guard > limit && lane == 0) atomicMin(&s_err, kInfoSelect);
    }
    __syncthreads();
    if (v_ < n) {
      const int u = suitor[v_];
      if (u > v_ && suitor[u] == v_) pairs[atomicAdd(&s_cnt, 1)] = make_int2(v_, u);
    }
    __syncthreads();
    if (s_err < 0) { info = s_err; break; }
    // rank the matched pairs by the record order; the first N_2 are the pivots
    const int cnt = s_cnt, sl = (cnt < it.n_2) ? cnt : it.n_2;
    for (int r = tid; r < cnt; r += THREADS) {
      const int2 a = pairs[r];
      const double wa = Ws[tri(a.x, a.y)];
      const unsigned ta = rtie(a.x, a.y);
      int k = 0;
      for (int o = 0; o < cnt; ++o) {
        const int2 b = pairs[o];
        if (rbetter(Ws[tri(b.x, b.y)], rtie(b.x, b.y), wa, ta)) ++k;
      }
      rk[k] = r;
    }
    __syncthreads();
    if (sl <= 0) { info = steps; break; }  // DSTEP_EXEC with SL = 0 (src/D/dstep.F90:421, 575-582)

    // ---- the 2x2 HSVDs of the pivots
    for (int r = tid; r < sl; r += THREADS) {
      const int2 a = pairs[rk[r]];
      const int p = a.x, q = a.y;
      const double *cp = As + pos[p] * lda, *cq = As + pos[q] * lda;
      double B[4] = { cp[p], cp[q], cq[p], cq[q] }, V[4], W[4];
      int inf = 0;
      dhsvd2(B, Jv[p], Jv[q], V, W, JK_TH1FIX, inf);
      BPiv x;
      x.p = p; x.q = q; x.info = inf; x.pad = 0;
      x.d0 = B[M11]; x.d1 = B[M22];
      if (inf >= 0) {
        if (inf & 2) {
          x.ba = rot_ba(V);
          const double Vt[4] = { V[M11], V[M12], V[M21], V[M22] };  // UT2, src/D/dtransf.F90:42-51
          x.tu = rot_ab(Vt);
        }
        if (inf & 4) x.tz = rot_ab(W);
        if ((inf & 1) && (inf & 6)) atomicAdd(&s_nl, 1);
      }
      else
        atomicMin(&s_err, inf);
      pv[r] = x;
    }
    __syncthreads();

    // ---- phase 1: rows p, q of A (BA); columns p, q of U (by V^T) and Z (by W)
    for (int k = tid; k < sl * n; k += THREADS) {
      const int r = k / n, j = k % n;
      const BPiv &x = pv[r];
      if (x.info < 0 || !(x.info & 2)) continue;
      double *c = As + j * lda;
      rot_apply(x.ba, c[x.p], c[x.q]);
    }
    for (int k = tid; k < sl * n; k += THREADS) {
      const int r = k / n, i = k % n;
      const BPiv &x = pv[r];
      if (x.info < 0) continue;
      if (x.info & 2) {
        double *u0 = U + (long long)x.p * n, *u1 = U + (long long)x.q * n;
        double a = u0[i], b = u1[i];
        rot_apply(x.tu, a, b);
        u0[i] = a; u1[i] = b;
      }
      if (x.info & 4) {
        double *z0 = Z + (long long)x.p * n, *z1 = Z + (long long)x.q * n;
        double a = z0[i], b = z1[i];
        rot_apply(x.tz, a, b);
        z0[i] = a; z1[i] = b;
      }
    }
    __syncthreads();
    const int err = s_err;
    if (err == 0) {
      // ---- phase 2: columns p, q of A (AB), then the diagonal write-back
      for (int k = tid; k < sl * n; k += THREADS) {
        const int r = k / n, i = k % n;
        const BPiv &x = pv[r];
        if (!(x.info & 4)) continue;
        rot_apply(x.tz, As[pos[x.p] * lda + i], As[pos[x.q] * lda + i]);
      }
      __syncthreads();
      for (int r = tid; r < sl; r += THREADS) {
        const BPiv &x = pv[r];
        if (x.info & 8) continue;
        double *cp = As + pos[x.p] * lda, *cq = As + pos[x.q] * lda;
        cp[x.p] = x.d0;
        cp[x.q] = 0.0;
        cq[x.p] = 0.0;
        cq[x.q] = x.d1;
      }
    }
    __syncthreads();
    const int nl = s_nl;
    if (s_learned && err == 0) {
      // ---- the scored ranking: the off-norm after the step (fixed summation order) and
      // the choice of the next step's ranking
      double acc = 0.0;
      for (int k = tid; k < n * n; k += THREADS) {
        const int i = k % n, j = k / n;
        if (i != j) {
          const double x = As[pos[j] * lda + i];
          acc = fma(x, x, acc);
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
      if ((tid & 31) == 0) s_red[tid >> 5] = acc;
      __syncthreads();
      if (tid == 0) {
        double off = 0.0;
        for (int w = 0; w < THREADS / 32; ++w) off += s_red[w];
        if (s_lstep && ((sl < nl) ? sl : nl) <= 0) {
          s_retry = 1;  // no effective pivot among the scored choices: an exact step decides
          s_lstep = 0;
          s_stall = 0;
        }
        else if (off > 16.0 * s_best) {
          s_learned = 0;  // the scored choices let the off-norm grow: the rest ranks exactly
          s_lstep = 0;
        }
        else {
          if (off < s_best) { s_best = off; s_stall = 0; }
          else s_stall += 1;
          if (s_stall >= stall_k) { s_lstep = 0; s_stall = 0; }
          else s_lstep = 1;
        }
      }
      __syncthreads();
    }
    // ---- the loop test
    if (err < 0) { info = err; break; }
    if (((sl < nl) ? sl : nl) <= 0) {
      if (s_retry) {
        __syncthreads();
        if (tid == 0) s_retry = 0;
        __syncthreads();
        continue;
      }
      info = steps;
      break;
    }
    ++steps;
    if (steps >= cap) { info = kInfoMaxSteps; break; }
    __syncthreads();
  }
  __syncthreads();

  // SIGMA, the zeroed diagonal, A back to global memory; Z := J Z^T J
  for (int k = tid; k < n * n; k += THREADS) {
    const int i = k % n, j = k / n;
    const double *c = As + pos[j] * lda;
    if (i == j) {
      gsigma[it.joff + i] = c[i];
      A[k] = 0.0;
    }
    else
      A[k] = c[i];
  }
  for (int k = tid; k < n * n; k += THREADS) {
    const int i = k % n, j = k / n;
    if (i >= j) continue;
    const double a = Z[(long long)j * n + i], b = Z[(long long)i * n + j];
    const bool flip = (Jv[i] != Jv[j]);
    Z[(long long)j * n + i] = flip ? -b : b;
    Z[(long long)i * n + j] = flip ? -a : a;
  }
  if (tid == 0) ginfo[it.index] = info;
  __syncthreads();
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1)
k_batch(const BatchItem *__restrict__ items, int count, int *counter, double *A, double *U, double *Z, const int *J,
        double *sigma, int *info, int nm, long long cap, int scored, int stall_k)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_m;
  for (;;) {
    if (threadIdx.x == 0) s_m = atomicAdd(counter, 1);
    __syncthreads();
    const int m = s_m;
    __syncthreads();
    if (m >= count) break;
    solve_one<THREADS>(items[m], A, U, Z, J, sigma, info, nm, cap, scored, stall_k, smem_raw);
  }
}

}  // namespace

size_t batch_smem(int nm) { return BLayout(nm).total; }

const int kBatchThreads[kBatchVariants] = { 256, 384, 512 };

cudaError_t batch_prepare(int nm)
{
  const int sm = (int)batch_smem(nm);
  cudaError_t e = cudaFuncSetAttribute(k_batch<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_batch<384>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_batch<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  return e;
}

int batch_blocks_per_sm(int variant, int nm)
{
  int b = 0;
  const size_t sm = batch_smem(nm);
  cudaError_t e;
  switch (variant) {
  case 0: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_batch<256>, 256, sm); break;
  case 1: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_batch<384>, 384, sm); break;
  default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_batch<512>, 512, sm); break;
  }
  if (e != cudaSuccess) { cudaGetLastError(); return 0; }
  return b;
}

cudaError_t launch_batch(int variant, int grid, const BatchItem *items, int count, int *counter, double *A, double *U,
                         double *Z, const int *J, double *sigma, int *info, int nm, long long cap, int scored, int stall_k,
                         cudaStream_t s)
{
  const size_t sm = batch_smem(nm);
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  switch (variant) {
  case 0: k_batch<256><<<grid, 256, sm, s>>>(items, count, counter, A, U, Z, J, sigma, info, nm, cap, scored, stall_k); break;
  case 1: k_batch<384><<<grid, 384, sm, s>>>(items, count, counter, A, U, Z, J, sigma, info, nm, cap, scored, stall_k); break;
  default: k_batch<512><<<grid, 512, sm, s>>>(items, count, counter, A, U, Z, J, sigma, info, nm, cap, scored, stall_k); break;
  }
  return cudaGetLastError();
}

}  // namespace jk
