// jk_api.cu -- the C ABI of libjkogb_b200.so (include/jkogb.h): device workspaces,
// the step-loop driver (CUDA graphs of whole steps, a device-side stop flag read
// back between graph launches) and the kernel-level entry points.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <vector>

#include "../../include/jkogb.h"
#include "jk_internal.h"

using namespace jk;

namespace {

thread_local long long g_launches = 0;

struct Guard {
  std::vector<void *> dev;
  void *pinned = nullptr;
  ~Guard()
  {
    for (void *p : dev) cudaFree(p);
    if (pinned) cudaFreeHost(pinned);
  }
  template <typename X> cudaError_t alloc(X **p, size_t bytes)
  {
    void *q = nullptr;
    const cudaError_t e = cudaMalloc(&q, bytes ? bytes : 16);
    if (e == cudaSuccess) { dev.push_back(q); *p = (X *)q; }
    return e;
  }
};

inline int cuda_fail(cudaError_t e)
{
  if (e == cudaErrorMemoryAllocation) { cudaGetLastError(); return JK_ERR_NOMEM; }
  fprintf(stderr, "libjkogb_b200: CUDA error %d (%s)\n", (int)e, cudaGetErrorString(e));
  cudaGetLastError();
  return JK_ERR_CUDA;
}

#define CK(x) do { const cudaError_t e_ = (x); if (e_ != cudaSuccess) return cuda_fail(e_); } while (0)

int max_order(int cplx)
{
  // k_rotate keeps two columns of A in shared memory and k_select its matching state
  // (227 KB per block each); the tie key packs p in 16 bits
  int n = (227 * 1024) / (2 * (cplx ? 16 : 8));
  while (n > 3 && (select_smem(n) > 227 * 1024 || colsort_e(n) > 16)) --n;
  return n < 65535 ? n : 65535;
}

// check the arguments as DSTEP_LOOP (src/D/dstep.F90:500-521) and DPROC_INIT / TRU do
int check_args(int n, int ldu, int lda, int ldz, const int *J, int n_2, int id_ncp, int id_tru, int cplx)
{
  if (n < 3) return -1;
  if (ldu < n) return -3;
  if (lda < n) return -5;
  if (ldz < n) return -7;
  if (n_2 < 0) return -16;
  if (id_ncp < 0 || id_ncp > 3) return JK_ERR_ID_NCP;
  if (id_ncp == 3 && n > kNcp3MaxN) return JK_ERR_TOO_LARGE;
  if (id_tru < 0 || id_tru > 2) return JK_ERR_ID_TRU;
  if (!J) return -8;
  for (int i = 0; i < n; ++i)
    if (J[i] != 1 && J[i] != -1) return JK_ERR_J;
  if (n > max_order(cplx)) return JK_ERR_TOO_LARGE;
  return 0;
}

// JSTEP_LEN, src/shared/jstep.F90:124-133
int jstep_len(int n, int n_2)
{
  if (!n_2) return (n / 2 > 0) ? n / 2 : 0;
  const int a = (n_2 > 0) ? n_2 : 0;
  return (a < n / 2) ? a : n / 2;
}

// device workspace of one solve
int make_workspace(Guard &g, Workspace &w, int n, int cplx, const int *J, int trace_on, int cap_steps, long long cap_piv)
{
  memset(&w, 0, sizeof(w));
  w.n = n;
  w.cplx = cplx;
  std::vector<int> plus, minus, j32(n);
  for (int i = 0; i < n; ++i) {
    j32[i] = J[i];
    (J[i] == 1 ? plus : minus).push_back(i);
  }
  w.n_plus = (int)plus.size();
  w.n_minus = (int)minus.size();
  const size_t pivsz = cplx ? sizeof(Piv<double2>) : sizeof(Piv<double>);
  const size_t rrsz = cplx ? sizeof(RowRot<double2>) : sizeof(RowRot<double>);
  const int half = n / 2 + 1;
  CK(g.alloc(&w.J, n * sizeof(int)));
  CK(g.alloc(&w.plus, (plus.size() + 1) * sizeof(int)));
  CK(g.alloc(&w.minus, (minus.size() + 1) * sizeof(int)));
  CK(g.alloc(&w.Wm, (size_t)n * n * sizeof(double)));
  if (cplx) CK(g.alloc(&w.mag, (size_t)n * n * sizeof(double)));
  CK(g.alloc(&w.piv, half * pivsz));
  CK(g.alloc(&w.rowrot, half * rrsz));
  CK(g.alloc(&w.list, (size_t)n * ((n + 7) & ~7) * sizeof(unsigned short)));
  CK(g.alloc(&w.rank, (size_t)n * n * sizeof(unsigned short)));
  CK(g.alloc(&w.len, n * sizeof(int)));
  CK(g.alloc(&w.unp, (n + 1) * sizeof(int)));
  CK(g.alloc(&w.st, sizeof(State)));
  if (trace_on) {
    const int cs = cap_steps > 0 ? cap_steps : 1;
    const long long cp = cap_piv > 0 ? cap_piv : 1;
    CK(g.alloc(&w.tr.sl, cs * sizeof(int)));
    CK(g.alloc(&w.tr.nl, cs * sizeof(int)));
    CK(g.alloc(&w.tr.trig, cs * sizeof(int)));
    CK(g.alloc(&w.tr.hyp, cs * sizeof(int)));
    CK(g.alloc(&w.tr.tw, cs * sizeof(double)));
    CK(g.alloc(&w.tr.rounds, cs * sizeof(int)));
    CK(g.alloc(&w.tr.piv, cp * sizeof(int2)));
  }
  CK(cudaMallocHost((void **)&g.pinned, sizeof(State)));
  w.st_host = (State *)g.pinned;
  CK(cudaMemcpy(w.J, j32.data(), n * sizeof(int), cudaMemcpyHostToDevice));
  if (!plus.empty()) CK(cudaMemcpy(w.plus, plus.data(), plus.size() * sizeof(int), cudaMemcpyHostToDevice));
  if (!minus.empty()) CK(cudaMemcpy(w.minus, minus.data(), minus.size() * sizeof(int), cudaMemcpyHostToDevice));
  State s0;
  memset(&s0, 0, sizeof(s0));
  s0.trace_on = trace_on;
  s0.trace_cap_steps = trace_on ? cap_steps : 0;
  s0.trace_cap_piv = trace_on ? cap_piv : 0;
  CK(cudaMemcpy(w.st, &s0, sizeof(State), cudaMemcpyHostToDevice));
  CK(prepare_kernels(n));
  return 0;
}

}  // namespace

// the learned ranking's network on the device
struct jk_scorer {
  Guard g;
  unsigned short *w = nullptr;  // BF16 weights
  float *b = nullptr;           // FP32 biases
  int nf = 0;
  int stall_k = 8;
};

// The step loop of DSTEP_LOOP / ZSTEP_LOOP (src/D/dstep.F90:564-583, src/Z/zstep.F90:575-594)
// on device buffers, resumable between steps: the workspace, the graph of `chunk`
// whole steps and the loop's position.
struct jk_solver {
  Guard g;
  Workspace w;
  jk_opts o;
  int n = 0, cplx = 0, n_2 = 0;
  int chunk = 32;                  // steps per graph launch; -1: plain stream launches
  cudaGraphExec_t exec = nullptr;  // the captured steps, for the buffers in `key`
  const void *key[4] = {};
  void *dA = nullptr, *dU = nullptr, *dZ = nullptr;
  cudaStream_t s = nullptr;
  int phase = 0;                   // 0 created, 1 running, 2 ended, 3 finished
  int info = 0;
  long long steps = 0;
  const jk_scorer *sc = nullptr;
  jk_trace *trace = nullptr;       // the internal callers' trace (copied out by finish)
  ~jk_solver()
  {
    if (exec) cudaGraphExecDestroy(exec);
  }
};

namespace {

int solver_make(jk_solver *v, int cplx, int n, const int *J, int n_2, int id_ncp, const jk_opts *opts,
                const jk_trace *trace, const jk_scorer *sc)
{
  memset(&v->o, 0, sizeof(v->o));
  if (opts) v->o = *opts;
  v->n = n;
  v->cplx = cplx;
  v->n_2 = jstep_len(n, n_2);
  v->sc = sc;
  v->chunk = (v->o.graph_steps == 0) ? 32 : v->o.graph_steps;
  Workspace &w = v->w;
  Guard &g = v->g;
  int rc = make_workspace(g, w, n, cplx, J, trace != nullptr, trace ? trace->max_steps : 0, trace ? trace->max_piv : 0);
  if (rc) return rc;
  w.zba_quirk = (v->o.zba_quirk == 0) ? 1 : 0;
  w.id_ncp = id_ncp;
  if (id_ncp == 3) {
    const size_t nn = (size_t)n * (n - 1) / 2;
    CK(g.alloc(&w.n3key, nn * sizeof(unsigned long long)));
    CK(g.alloc(&w.n3tie, nn * sizeof(unsigned)));
    CK(g.alloc(&w.n3sorted, nn * sizeof(int)));
    CK(g.alloc(&w.n3val, nn * sizeof(double)));
    CK(g.alloc(&w.n3len, nn * sizeof(int)));
    CK(g.alloc(&w.n3it, sizeof(int)));
    CK(cudaMemset(w.n3it, 0, sizeof(int)));
  }
  if (sc) {
    // a learned solve: the scorer's device parameters, the off-norm buffers
    w.learned = 1;
    w.sc.w = sc->w;
    w.sc.b = sc->b;
    w.sc.nf = sc->nf;
    CK(g.alloc(&w.offpart, kOffBlocks * sizeof(double)));
    CK(g.alloc(&w.offcount, sizeof(int)));
    CK(cudaMemset(w.offcount, 0, sizeof(int)));
    // the Gram form of the scanned weights: the "+" x "-" column products, the column norms
    CK(g.alloc(&w.gram, ((size_t)(cplx ? 2 : 1) * w.n_plus * w.n_minus + 1) * sizeof(double)));
    CK(g.alloc(&w.cn, (size_t)n * sizeof(double)));
    CK(prepare_gram());
  }
  return 0;
}

// kernel launches of one step of this solve
long long step_launches(const Workspace &w)
{
  const bool hyp = (w.n_plus > 0 && w.n_minus > 0);
  const int learned = !w.learned ? 0 : (hyp ? 4 : 1);  // norms, Gram, weights; the off-norm
  return kStepLaunches - (hyp ? 0 : 1) + ((w.cplx && hyp) ? 1 : 0) + learned;
}

// a new solve (dsigma NULL), or the continuation of a loop that ended after steps0
// steps with A, U, Z, SIGMA as its end left them
int solver_start(jk_solver *v, void *dU, void *dA, void *dZ, const double *dsigma, long long steps0, cudaStream_t s)
{
  if (steps0 < 0 || steps0 > 0x7FFFFFFF) return -6;
  v->dA = dA;
  v->dU = dU;
  v->dZ = dZ;
  v->s = s;
  v->phase = 1;
  v->info = 0;
  v->steps = steps0;
  g_launches = 2;  // state init, U = Z = I (or the two kernels that undo the loop's end)
  if (dsigma) CK(launch_unfinish(v->w, dA, dZ, dsigma, s));
  CK(launch_init(v->w, dU, dZ, v->sc ? 1 : 0, v->sc ? v->sc->stall_k : 0, (int)steps0, dsigma ? 0 : 1, s));
  if (v->w.n3it) CK(cudaMemsetAsync(v->w.n3it, 0, sizeof(int), s));
  if (v->w.offcount) CK(cudaMemsetAsync(v->w.offcount, 0, sizeof(int), s));
  return 0;
}

// capture `chunk` whole steps as a graph for the current buffers and stream; if capture
// fails, the loop uses plain stream launches
void solver_graph(jk_solver *v)
{
  const void *key[4] = { v->dA, v->dU, v->dZ, v->s };
  if (v->chunk <= 0) return;
  if (v->exec && !memcmp(key, v->key, sizeof(key))) return;
  if (v->exec) { cudaGraphExecDestroy(v->exec); v->exec = nullptr; }
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamBeginCapture(v->s, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    for (int k = 0; k < v->chunk && e == cudaSuccess; ++k) e = launch_step(v->w, v->dA, v->dU, v->dZ, v->n_2, v->s);
    const cudaError_t e2 = cudaStreamEndCapture(v->s, &graph);
    if (e == cudaSuccess) e = e2;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&v->exec, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (v->exec) { cudaGraphExecDestroy(v->exec); v->exec = nullptr; }
    v->chunk = -1;
  }
  memcpy(v->key, key, sizeof(key));
}

int solver_advance(jk_solver *v, long long k)
{
  if (v->phase == 0 || v->phase == 3) return JK_ERR_STATE;
  if (v->phase == 2) return 1;
  // the step count at which the loop waits: the caller's slice, capped by max_steps
  long long target = (k > 0) ? v->steps + k : 0;
  if (v->o.max_steps > 0 && (target == 0 || target > v->o.max_steps)) target = v->o.max_steps;
  CK(launch_limit(v->w, target, v->s));
  ++g_launches;
  solver_graph(v);
  const int per_sync = (v->chunk > 0) ? v->chunk : 32;
  const long long per_step = step_launches(v->w);
  long long last = v->steps;
  int idle = 0;
  for (;;) {
    cudaError_t e = cudaSuccess;
    if (v->exec) e = cudaGraphLaunch(v->exec, v->s);
    else
      for (int j = 0; j < per_sync && e == cudaSuccess; ++j) e = launch_step(v->w, v->dA, v->dU, v->dZ, v->n_2, v->s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(v->w.st_host, v->w.st, sizeof(State), cudaMemcpyDeviceToHost, v->s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(v->s);
    if (e != cudaSuccess) return cuda_fail(e);
    g_launches += (long long)per_sync * per_step;
    const State &h = *v->w.st_host;
    v->steps = h.steps;
    if (h.stop == 1) { v->phase = 2; v->info = h.info; return 1; }
    if (h.stop == 2) {
      if (v->o.max_steps > 0 && v->steps >= v->o.max_steps) { v->phase = 2; v->info = JK_ERR_MAX_STEPS; return 1; }
      return 0;
    }
    // every graph launch takes at least one step or ends the loop (a learned step
    // without an effective pivot is followed by an exact one)
    if (v->steps == last) {
      if (++idle >= 3) return JK_ERR_STALL;
    }
    else { idle = 0; last = v->steps; }
  }
}

int solver_finish(jk_solver *v, double *dsigma, int *exact_steps)
{
  if (v->phase == 0 || v->phase == 3) return JK_ERR_STATE;
  const int info = (v->phase == 2) ? v->info : JK_ERR_MAX_STEPS;
  v->phase = 3;
  cudaStream_t s = v->s;
  Workspace &w = v->w;
  g_launches += 2;  // sigma, J Z^T J
  CK(launch_finish(w, v->dA, v->dZ, dsigma, s));
  CK(cudaMemcpyAsync(w.st_host, w.st, sizeof(State), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (exact_steps) *exact_steps = w.st_host->exact_steps;
  jk_trace *trace = v->trace;
  if (trace) {
    const State &h = *w.st_host;
    const int ns = h.trace_steps < trace->max_steps ? h.trace_steps : trace->max_steps;
    trace->n_steps = h.trace_steps;
    if (ns > 0) {
      if (trace->sl) CK(cudaMemcpyAsync(trace->sl, w.tr.sl, ns * sizeof(int), cudaMemcpyDeviceToHost, s));
      if (trace->nl) CK(cudaMemcpyAsync(trace->nl, w.tr.nl, ns * sizeof(int), cudaMemcpyDeviceToHost, s));
      if (trace->trig) CK(cudaMemcpyAsync(trace->trig, w.tr.trig, ns * sizeof(int), cudaMemcpyDeviceToHost, s));
      if (trace->hyp) CK(cudaMemcpyAsync(trace->hyp, w.tr.hyp, ns * sizeof(int), cudaMemcpyDeviceToHost, s));
      if (trace->tw) CK(cudaMemcpyAsync(trace->tw, w.tr.tw, ns * sizeof(double), cudaMemcpyDeviceToHost, s));
      if (trace->rounds) CK(cudaMemcpyAsync(trace->rounds, w.tr.rounds, ns * sizeof(int), cudaMemcpyDeviceToHost, s));
    }
    const long long np = h.trace_npiv < trace->max_piv ? h.trace_npiv : trace->max_piv;
    trace->n_piv = np;
    if (np > 0 && trace->piv) {
      CK(cudaMemcpyAsync(trace->piv, w.tr.piv, np * sizeof(int2), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      for (long long k = 0; k < 2 * np; ++k) trace->piv[k] += 1;
    }
  }
  CK(cudaStreamSynchronize(s));
  return info;
}

// the loop of DSTEP_LOOP / ZSTEP_LOOP on device buffers, in one call
int run_loop(int cplx, int n, void *dU, void *dA, void *dZ, const int *J, double *dsigma, int n_2, int id_ncp, int id_tru,
             const jk_opts *opts, jk_trace *trace, cudaStream_t s, const jk_scorer *sc = nullptr, int *exact_steps = nullptr)
{
  (void)id_tru;  // the pair order does not change the sorted records
  jk_solver v;
  int rc = solver_make(&v, cplx, n, J, n_2, id_ncp, opts, trace, sc);
  if (rc) return rc;
  v.trace = trace;
  if ((rc = solver_start(&v, dU, dA, dZ, nullptr, 0, s))) return rc;
  rc = solver_advance(&v, 0);
  if (rc < 0) return rc;
  return solver_finish(&v, dsigma, exact_steps);
}

// a device buffer argument: not NULL and aligned as the kernels read it (8 bytes for real
// data; 16 for complex data, and for A of a scored real solve, whose Gram kernel copies 16
// bytes at a time)
bool dev_ok(const void *p, size_t align) { return p && !((uintptr_t)p & (uintptr_t)(align - 1)); }

// the device matrices of a loop entry, reported by their position in DSTEP_LOOP's argument
// list (src/D/dstep.F90:472-482: U 2, A 4, Z 6; SIGMA is 9), as its INFO reports bad arguments
int check_dev(int cplx, int scored, const void *dU, const void *dA, const void *dZ)
{
  const size_t m = cplx ? 16 : 8;
  if (!dev_ok(dU, m)) return -2;
  if (!dev_ok(dA, (cplx || scored) ? 16 : 8)) return -4;
  if (!dev_ok(dZ, m)) return -6;
  return 0;
}

int pick_device(const jk_opts *opts)
{
  int cnt = 0;
  if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt <= 0) { cudaGetLastError(); return JK_ERR_NO_DEVICE; }
  if (opts && opts->device > 0) {
    if (opts->device >= cnt) return JK_ERR_NO_DEVICE;
    if (cudaSetDevice(opts->device) != cudaSuccess) return JK_ERR_CUDA;
  }
  return 0;
}

// host-buffer form: copy in (leading dimensions honoured), run, copy out
int host_loop(int cplx, int n, double *U, int ldu, double *A, int lda, double *Z, int ldz, const int *J, double *sigma,
              int n_2, int id_ncp, int id_tru, const jk_opts *opts, jk_trace *trace)
{
  int rc = check_args(n, ldu, lda, ldz, J, n_2, id_ncp, id_tru, cplx);
  if (rc) return rc;
  if ((rc = pick_device(opts))) return rc;
  const size_t es = cplx ? 16 : 8;
  Guard g;
  void *dA, *dU, *dZ;
  double *ds;
  CK(g.alloc(&dA, (size_t)n * n * es));
  CK(g.alloc(&dU, (size_t)n * n * es));
  CK(g.alloc(&dZ, (size_t)n * n * es));
  CK(g.alloc(&ds, n * sizeof(double)));
  cudaStream_t s;
  CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  CK(cudaMemcpy2DAsync(dA, n * es, A, (size_t)lda * es, n * es, n, cudaMemcpyHostToDevice, s));
  const int info = run_loop(cplx, n, dU, dA, dZ, J, ds, n_2, id_ncp, id_tru, opts, trace, s);
  if (info > JK_ERR_CUDA || info < JK_ERR_NO_DEVICE) {
    CK(cudaMemcpy2DAsync(A, (size_t)lda * es, dA, n * es, n * es, n, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpy2DAsync(U, (size_t)ldu * es, dU, n * es, n * es, n, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpy2DAsync(Z, (size_t)ldz * es, dZ, n * es, n * es, n, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(sigma, ds, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  CK(cudaStreamSynchronize(s));
  cudaStreamDestroy(s);
  return info;
}

}  // namespace

extern "C" {

int jk_dstep_loop(int n, double *U, int ldu, double *A, int lda, double *Z, int ldz, const int *J, double *sigma, int n_2,
                  int id_ncp, int id_tru, const jk_opts *opts, jk_trace *trace)
{
  return host_loop(0, n, U, ldu, A, lda, Z, ldz, J, sigma, n_2, id_ncp, id_tru, opts, trace);
}

int jk_zstep_loop(int n, double *U, int ldu, double *A, int lda, double *Z, int ldz, const int *J, double *sigma, int n_2,
                  int id_ncp, int id_tru, const jk_opts *opts, jk_trace *trace)
{
  return host_loop(1, n, U, ldu, A, lda, Z, ldz, J, sigma, n_2, id_ncp, id_tru, opts, trace);
}

int jk_dstep_loop_dev(int n, double *dU, double *dA, double *dZ, const int *J, double *dsigma, int n_2, int id_ncp, int id_tru,
                      const jk_opts *opts, jk_trace *trace, void *stream)
{
  int rc = check_args(n, n, n, n, J, n_2, id_ncp, id_tru, 0);
  if (!rc) rc = check_dev(0, 0, dU, dA, dZ);
  if (!rc && !dev_ok(dsigma, 8)) rc = -9;
  if (rc) return rc;
  return run_loop(0, n, dU, dA, dZ, J, dsigma, n_2, id_ncp, id_tru, opts, trace, (cudaStream_t)stream);
}

int jk_zstep_loop_dev(int n, double *dU, double *dA, double *dZ, const int *J, double *dsigma, int n_2, int id_ncp, int id_tru,
                      const jk_opts *opts, jk_trace *trace, void *stream)
{
  int rc = check_args(n, n, n, n, J, n_2, id_ncp, id_tru, 1);
  if (!rc) rc = check_dev(1, 0, dU, dA, dZ);
  if (!rc && !dev_ok(dsigma, 8)) rc = -9;
  if (rc) return rc;
  return run_loop(1, n, dU, dA, dZ, J, dsigma, n_2, id_ncp, id_tru, opts, trace, (cudaStream_t)stream);
}

jk_solver *jk_solver_create(int n, int complex_, const int *J, int n_2, int id_ncp, int id_tru, const jk_opts *opts,
                            int *info)
{
  const int cplx = complex_ ? 1 : 0;
  int rc = check_args(n, n, n, n, J, n_2, id_ncp, id_tru, cplx);
  jk_solver *v = nullptr;
  if (!rc) {
    v = new jk_solver;
    rc = solver_make(v, cplx, n, J, n_2, id_ncp, opts, nullptr, nullptr);
    if (rc) { delete v; v = nullptr; }
  }
  if (info) *info = rc;
  return v;
}

void jk_solver_destroy(jk_solver *v) { delete v; }

int jk_solver_begin(jk_solver *v, double *dU, double *dA, double *dZ, void *stream)
{
  if (!v) return -1;
  if (check_dev(v->cplx, 0, dU, dA, dZ)) return -2;
  return solver_start(v, dU, dA, dZ, nullptr, 0, (cudaStream_t)stream);
}

int jk_solver_resume(jk_solver *v, double *dU, double *dA, double *dZ, const double *dsigma, long long steps, void *stream)
{
  if (!v) return -1;
  if (!dev_ok(dsigma, 8) || check_dev(v->cplx, 0, dU, dA, dZ)) return -2;
  // a complex loop's end keeps only the real parts of the diagonal in SIGMA
  if (v->cplx) return JK_ERR_STATE;
  return solver_start(v, dU, dA, dZ, dsigma, steps, (cudaStream_t)stream);
}

int jk_solver_advance(jk_solver *v, long long steps)
{
  if (!v) return -1;
  if (steps < 0) return -2;
  return solver_advance(v, steps);
}

long long jk_solver_steps(const jk_solver *v) { return v ? v->steps : -1; }

int jk_solver_finish(jk_solver *v, double *dsigma)
{
  if (!v) return -1;
  if (!dev_ok(dsigma, 8)) return -2;
  return solver_finish(v, dsigma, nullptr);
}

static int hsvd2_batch(int cplx, int count, double *A, const int *J, double *U, double *Z, int *info, double th1)
{
  if (count < 0) return -1;
  if (!count) return 0;
  int rc = pick_device(nullptr);
  if (rc) return rc;
  const size_t bs = 4 * (cplx ? 16 : 8) * (size_t)count;
  Guard g;
  void *dA, *dU, *dZ;
  int *dJ, *di;
  CK(g.alloc(&dA, bs));
  CK(g.alloc(&dU, bs));
  CK(g.alloc(&dZ, bs));
  CK(g.alloc(&dJ, 2 * sizeof(int) * (size_t)count));
  CK(g.alloc(&di, sizeof(int) * (size_t)count));
  CK(cudaMemcpy(dA, A, bs, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dJ, J, 2 * sizeof(int) * (size_t)count, cudaMemcpyHostToDevice));
  CK(launch_hsvd2_batch(cplx, count, dA, dJ, dU, dZ, di, th1, 0));
  CK(cudaMemcpy(A, dA, bs, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(U, dU, bs, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(Z, dZ, bs, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(info, di, sizeof(int) * (size_t)count, cudaMemcpyDeviceToHost));
  return 0;
}

int jk_dhsvd2_batch(int count, double *A, const int *J, double *U, double *Z, int *info, double th1)
{
  return hsvd2_batch(0, count, A, J, U, Z, info, th1);
}

int jk_zhsvd2_batch(int count, double *A, const int *J, double *U, double *Z, int *info, double th1)
{
  return hsvd2_batch(1, count, A, J, U, Z, info, th1);
}

static int weights(int cplx, int n, const double *A, int lda, const int *J, double *W)
{
  int rc = check_args(n, n, lda, n, J, 0, 0, 0, cplx);
  if (rc) return rc;
  if ((rc = pick_device(nullptr))) return rc;
  const size_t es = cplx ? 16 : 8;
  Guard g;
  Workspace w;
  rc = make_workspace(g, w, n, cplx, J, 0, 0, 0);
  if (rc) return rc;
  void *dA;
  CK(g.alloc(&dA, (size_t)n * n * es));
  CK(cudaMemcpy2D(dA, n * es, A, (size_t)lda * es, n * es, n, cudaMemcpyHostToDevice));
  CK(cudaMemset(w.Wm, 0xFF, (size_t)n * n * sizeof(double)));  // all-ones bits: a NaN on the diagonal
  CK(launch_weights(w, dA, 0));
  CK(cudaMemcpy(W, w.Wm, (size_t)n * n * sizeof(double), cudaMemcpyDeviceToHost));
  return 0;
}

int jk_dweights(int n, const double *A, int lda, const int *J, double *W) { return weights(0, n, A, lda, J, W); }
int jk_zweights(int n, const double *A, int lda, const int *J, double *W) { return weights(1, n, A, lda, J, W); }

int jk_select(int n, const double *W, int n_2, int *piv)
{
  if (n < 2) return -1;
  if (n_2 < 0) return -16;
  if (n > 65535) return JK_ERR_TOO_LARGE;
  int rc = pick_device(nullptr);
  if (rc) return rc;
  n_2 = jstep_len(n, n_2);
  std::vector<int> J(n, 1);
  Guard g;
  Workspace w;
  rc = make_workspace(g, w, n, 0, J.data(), 0, 0, 0);
  if (rc) return rc;
  CK(cudaMemcpy(w.Wm, W, (size_t)n * n * sizeof(double), cudaMemcpyHostToDevice));
  CK(launch_match(w, n_2, 0));
  CK(cudaMemcpy(w.st_host, w.st, sizeof(State), cudaMemcpyDeviceToHost));
  const int sl = w.st_host->sl;
  std::vector<Piv<double>> pv(sl > 0 ? sl : 1);
  if (sl > 0) CK(cudaMemcpy(pv.data(), w.piv, sl * sizeof(Piv<double>), cudaMemcpyDeviceToHost));
  for (int i = 0; i < sl; ++i) { piv[2 * i] = pv[i].p + 1; piv[2 * i + 1] = pv[i].q + 1; }
  return sl;
}

struct jk_handle {
  Guard g;
  Workspace w;
};

jk_handle *jk_handle_create(int n, int complex_, const int *J, int *info)
{
  int rc = check_args(n, n, n, n, J, 0, 0, 0, complex_ ? 1 : 0);
  if (!rc) rc = pick_device(nullptr);
  jk_handle *h = nullptr;
  if (!rc) {
    h = new jk_handle;
    rc = make_workspace(h->g, h->w, n, complex_ ? 1 : 0, J, 0, 0, 0);
    if (rc) { delete h; h = nullptr; }
  }
  if (info) *info = rc;
  return h;
}

void jk_handle_destroy(jk_handle *h) { delete h; }

int jk_handle_weights(jk_handle *h, const double *dA, double *dW, void *stream)
{
  if (!h || !dev_ok(dA, h->w.cplx ? 16 : 8)) return -1;
  cudaStream_t s = (cudaStream_t)stream;
  CK(launch_weights(h->w, dA, s));
  if (dW) CK(cudaMemcpyAsync(dW, h->w.Wm, (size_t)h->w.n * h->w.n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  return 0;
}

// Weights with no device allocation; scratch in a static device array (jk_kernels.cu).
int jk_dweights_noalloc(int n, const double *dA, const int *J, double *dW, void *stream)
{
  static_assert(JK_NOALLOC_MAX_N == kNoallocMaxN, "header and library disagree on the scratch size");
  if (n < 3) return -1;
  if (n > JK_NOALLOC_MAX_N) return JK_ERR_SCRATCH;
  if (!dA) return -2;
  if (!J) return -8;
  if (!dW) return -4;
  for (int i = 0; i < n; ++i)
    if (J[i] != 1 && J[i] != -1) return JK_ERR_J;
  int rc = pick_device(nullptr);
  if (rc) return rc;
  CK(launch_weights_noalloc(n, dA, J, dW, (cudaStream_t)stream));
  return 0;
}

// ---------------------------------------------------------------------------
// the batched solver: many small real matrices, one persistent launch (jk_batch.cu)
// ---------------------------------------------------------------------------
struct jk_batch {
  Guard g;
  int count = 0, nm = 0, variant = kBatchVariants - 1, grid = 0;
  long long cap = 0, total = 0, totaln = 0;
  BatchItem *items = nullptr;
  int *counter = nullptr, *J = nullptr;
  cudaGraphExec_t exec = nullptr;
  const void *key[6] = {};  // the buffers and stream the graph was captured with
  int key_variant = -1, key_scored = -1;
  int scored = 0, stall_k = 8;  // the Gram-form ranking (jk_batch_set_scorer)
  ~jk_batch()
  {
    if (exec) cudaGraphExecDestroy(exec);
  }
};

static int batch_grid(int variant, int nm)
{
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return sms * batch_blocks_per_sm(variant, nm);
}

jk_batch *jk_batch_create(int count, const int *n, const int *n_2, const int *J, const jk_opts *opts, int *info)
{
  int rc = 0;
  if (count < 1) rc = -1;
  else if (!n) rc = -2;
  else if (!n_2) rc = -3;
  else if (!J) rc = -4;
  long long total = 0, totaln = 0;
  int nm = 0;
  for (int m = 0; !rc && m < count; ++m) {
    if (n[m] < 3) rc = -2;
    else if (n[m] > JK_BATCH_MAX_N) rc = JK_ERR_TOO_LARGE;
    else if (n_2[m] < 0) rc = -3;
    for (int i = 0; !rc && i < n[m]; ++i)
      if (J[totaln + i] != 1 && J[totaln + i] != -1) rc = JK_ERR_J;
    if (!rc) {
      total += (long long)n[m] * n[m];
      totaln += n[m];
      nm = (n[m] > nm) ? n[m] : nm;
    }
  }
  if (!rc) rc = pick_device(opts);
  jk_batch *b = nullptr;
  if (!rc) {
    b = new jk_batch;
    b->count = count;
    b->nm = nm;
    b->total = total;
    b->totaln = totaln;
    b->cap = (opts && opts->max_steps > 0) ? opts->max_steps : JK_BATCH_STEP_BOUND(nm);
    // the work order: largest matrices first (the cost grows as N^4)
    std::vector<BatchItem> it(count);
    long long off = 0;
    int joff = 0;
    for (int m = 0; m < count; ++m) {
      it[m].off = off;
      it[m].n = n[m];
      it[m].n_2 = jstep_len(n[m], n_2[m]);
      it[m].joff = joff;
      it[m].index = m;
      off += (long long)n[m] * n[m];
      joff += n[m];
    }
    std::stable_sort(it.begin(), it.end(), [](const BatchItem &x, const BatchItem &y) { return x.n > y.n; });
    auto fail = [&](cudaError_t e) { rc = cuda_fail(e); };
    cudaError_t e = b->g.alloc(&b->items, count * sizeof(BatchItem));
    if (e == cudaSuccess) e = b->g.alloc(&b->counter, sizeof(int));
    if (e == cudaSuccess) e = b->g.alloc(&b->J, totaln * sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(b->items, it.data(), count * sizeof(BatchItem), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->J, J, totaln * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = batch_prepare(nm);
    if (e != cudaSuccess) fail(e);
    if (!rc) {
      b->grid = batch_grid(b->variant, nm);
      if (b->grid <= 0) rc = JK_ERR_CUDA;
    }
    if (rc) { delete b; b = nullptr; }
  }
  if (info) *info = rc;
  return b;
}

void jk_batch_destroy(jk_batch *b) { delete b; }

int jk_batch_run(jk_batch *b, double *dA, double *dU, double *dZ, double *dsigma, int *dinfo, void *stream)
{
  if (!b || !dev_ok(dA, 8) || !dev_ok(dU, 8) || !dev_ok(dZ, 8) || !dev_ok(dsigma, 8) || !dev_ok(dinfo, 4)) return -1;
  cudaStream_t s = (cudaStream_t)stream;
  const void *key[6] = { dA, dU, dZ, dsigma, dinfo, stream };
  bool same = (b->exec != nullptr) && (b->key_variant == b->variant) && (b->key_scored == b->scored);
  for (int k = 0; k < 6; ++k) same = same && (key[k] == b->key[k]);
  if (!same) {
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    // capture the launch (counter reset + persistent kernel) once per set of buffers
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      const cudaError_t e1 = launch_batch(b->variant, b->grid, b->items, b->count, b->counter, dA, dU, dZ, b->J, dsigma,
                                          dinfo, b->nm, b->cap, b->scored, b->stall_k, s);
      const cudaError_t e2 = cudaStreamEndCapture(s, &graph);
      e = (e1 != cudaSuccess) ? e1 : e2;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      cudaGetLastError();
      b->exec = nullptr;
      g_launches = 1;
      CK(launch_batch(b->variant, b->grid, b->items, b->count, b->counter, dA, dU, dZ, b->J, dsigma, dinfo, b->nm,
                      b->cap, b->scored, b->stall_k, s));
      return 0;
    }
    for (int k = 0; k < 6; ++k) b->key[k] = key[k];
    b->key_variant = b->variant;
    b->key_scored = b->scored;
  }
  g_launches = 1;
  CK(cudaGraphLaunch(b->exec, s));
  return 0;
}

int jk_batch_set_scorer(jk_batch *b, const jk_scorer *sc)
{
  if (!b) return -1;
  if (sc && sc->nf != 0) return -2;  // the batched kernel ranks by the Gram form only
  b->scored = sc ? 1 : 0;
  b->stall_k = sc ? sc->stall_k : 8;
  return 0;
}

int jk_batch_tune(jk_batch *b, const double *dA, double *dU, double *dZ, double *dsigma, int *dinfo, void *stream)
{
  if (!b || !dev_ok(dA, 8) || !dev_ok(dU, 8) || !dev_ok(dZ, 8) || !dev_ok(dsigma, 8) || !dev_ok(dinfo, 4)) return -1;
  cudaStream_t s = (cudaStream_t)stream;
  Guard g;
  double *scratch = nullptr;
  CK(g.alloc(&scratch, b->total * sizeof(double)));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  float best_ms = -1.0f;
  int best = b->variant;
  cudaError_t err = cudaSuccess;
  // time a bounded sample: the first (largest) matrices of the work order, two per
  // resident block, each stopped after at most 30 N steps
  const long long cap_t = (b->cap < 30LL * b->nm) ? b->cap : 30LL * b->nm;
  for (int v = 0; v < kBatchVariants && err == cudaSuccess; ++v) {
    const int grid = batch_grid(v, b->nm);
    if (grid <= 0) continue;
    const int sub = (b->count < 2 * grid) ? b->count : 2 * grid;
    err = cudaMemcpyAsync(scratch, dA, b->total * sizeof(double), cudaMemcpyDeviceToDevice, s);
    if (err == cudaSuccess) err = cudaEventRecord(e0, s);
    if (err == cudaSuccess)
      err = launch_batch(v, grid, b->items, sub, b->counter, scratch, dU, dZ, b->J, dsigma, dinfo, b->nm, cap_t, b->scored,
                         b->stall_k, s);
    if (err == cudaSuccess) err = cudaEventRecord(e1, s);
    if (err == cudaSuccess) err = cudaEventSynchronize(e1);
    float ms = 0.0f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    if (err == cudaSuccess && (best_ms < 0.0f || ms < best_ms)) { best_ms = ms; best = v; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess) return cuda_fail(err);
  b->variant = best;
  b->grid = batch_grid(best, b->nm);
  return kBatchThreads[best];
}

int jk_dstep_loop_batched(int count, const int *n, const int *n_2, double *A, double *U, double *Z, const int *J,
                          double *sigma, int *info, const jk_opts *opts)
{
  if (!A || !U || !Z || !sigma || !info) return -5;
  int rc = 0;
  jk_batch *b = jk_batch_create(count, n, n_2, J, opts, &rc);
  if (!b) return rc;
  Guard g;
  double *dA = nullptr, *dU = nullptr, *dZ = nullptr, *ds = nullptr;
  int *di = nullptr;
  cudaStream_t s = nullptr;
  auto body = [&]() -> int {
    CK(g.alloc(&dA, b->total * sizeof(double)));
    CK(g.alloc(&dU, b->total * sizeof(double)));
    CK(g.alloc(&dZ, b->total * sizeof(double)));
    CK(g.alloc(&ds, b->totaln * sizeof(double)));
    CK(g.alloc(&di, count * sizeof(int)));
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    CK(cudaMemcpyAsync(dA, A, b->total * sizeof(double), cudaMemcpyHostToDevice, s));
    const int r = jk_batch_run(b, dA, dU, dZ, ds, di, s);
    if (r) return r;
    CK(cudaMemcpyAsync(A, dA, b->total * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(U, dU, b->total * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(Z, dZ, b->total * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(sigma, ds, b->totaln * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(info, di, count * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return 0;
  };
  rc = body();
  if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
  if (s) cudaStreamDestroy(s);
  jk_batch_destroy(b);
  return rc;
}

// ---------------------------------------------------------------------------
// the learned ranking: scorer objects, the scored loop, training kernels
// ---------------------------------------------------------------------------
int jk_mlp_nparams(int nf) { return (nf == kMlpFeat) ? mlp_params(nf) : -1; }

jk_scorer *jk_scorer_create(int nf, const float *params, int stall_k, int *info)
{
  int rc = 0;
  if (nf != kMlpFeat && nf != 0) rc = -1;
  else if (nf && !params) rc = -2;
  else if (stall_k < 1) rc = -3;
  if (!rc) rc = pick_device(nullptr);
  jk_scorer *sc = nullptr;
  if (!rc && nf == 0) {
    // the Gram-guided ranking: no network
    sc = new jk_scorer;
    sc->nf = 0;
    sc->stall_k = stall_k;
  }
  else if (!rc) {
    sc = new jk_scorer;
    sc->nf = nf;
    sc->stall_k = stall_k;
    const int np = mlp_params(nf);
    float *tmp = nullptr;
    Guard g;
    cudaError_t e = g.alloc(&tmp, np * sizeof(float));
    if (e == cudaSuccess) e = sc->g.alloc(&sc->w, (kMlpHidden * nf + kMlpHidden * kMlpHidden + kMlpHidden) * sizeof(unsigned short));
    if (e == cudaSuccess) e = sc->g.alloc(&sc->b, (2 * kMlpHidden + 1) * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(tmp, params, np * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = mlp_pack(nf, tmp, sc->w, sc->b, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) { rc = cuda_fail(e); delete sc; sc = nullptr; }
  }
  if (info) *info = rc;
  return sc;
}

void jk_scorer_destroy(jk_scorer *sc) { delete sc; }

int jk_dstep_loop_dev_scored(int n, double *dU, double *dA, double *dZ, const int *J, double *dsigma, int n_2,
                             const jk_scorer *sc, const jk_opts *opts, jk_trace *trace, int *exact_steps, void *stream)
{
  if (!sc) return -9;
  int rc = check_args(n, n, n, n, J, n_2, 0, 0, 0);
  if (!rc) rc = check_dev(0, 1, dU, dA, dZ);
  if (!rc && !dev_ok(dsigma, 8)) rc = -9;
  if (rc) return rc;
  return run_loop(0, n, dU, dA, dZ, J, dsigma, n_2, 0, 0, opts, trace, (cudaStream_t)stream, sc, exact_steps);
}

int jk_zstep_loop_dev_scored(int n, double *dU, double *dA, double *dZ, const int *J, double *dsigma, int n_2,
                             const jk_scorer *sc, const jk_opts *opts, jk_trace *trace, int *exact_steps, void *stream)
{
  if (!sc) return -9;
  int rc = check_args(n, n, n, n, J, n_2, 0, 0, 1);
  if (!rc) rc = check_dev(1, 1, dU, dA, dZ);
  if (!rc && !dev_ok(dsigma, 8)) rc = -9;
  if (rc) return rc;
  return run_loop(1, n, dU, dA, dZ, J, dsigma, n_2, 0, 0, opts, trace, (cudaStream_t)stream, sc, exact_steps);
}

static long long features(int cplx, int n, const double *dA, const int *J, int step, float *dX, double *dWg,
                          void *stream)
{
  if (n < 3 || !dev_ok(dA, 16) || !J || !dX) return -1;
  std::vector<int> plus, minus;
  for (int i = 0; i < n; ++i) {
    if (J[i] == 1) plus.push_back(i);
    else if (J[i] == -1) minus.push_back(i);
    else return JK_ERR_J;
  }
  const long long cnt = (long long)plus.size() * (long long)minus.size();
  if (!cnt) return 0;
  Guard g;
  int *dp = nullptr, *dm = nullptr;
  double *G = nullptr, *cn = nullptr;
  State *st = nullptr;
  cudaStream_t s = (cudaStream_t)stream;
  CK(g.alloc(&dp, plus.size() * sizeof(int)));
  CK(g.alloc(&dm, minus.size() * sizeof(int)));
  CK(g.alloc(&G, (cplx ? 2 : 1) * cnt * sizeof(double)));
  CK(g.alloc(&cn, n * sizeof(double)));
  CK(g.alloc(&st, sizeof(State)));
  State s0;
  memset(&s0, 0, sizeof(s0));
  s0.learned = s0.learned_step = 1;  // the Gram kernels run in scored steps only
  CK(cudaMemcpy(st, &s0, sizeof(State), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dp, plus.data(), plus.size() * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dm, minus.data(), minus.size() * sizeof(int), cudaMemcpyHostToDevice));
  CK(mlp_features(cplx, n, dA, dp, dm, (int)plus.size(), (int)minus.size(), step, st, G, cn, dX, dWg, s));
  CK(cudaStreamSynchronize(s));  // the temporaries are freed on return
  return cnt;
}

long long jk_mlp_features(int n, const double *dA, const int *J, int step, float *dX, double *dWg, void *stream)
{
  return features(0, n, dA, J, step, dX, dWg, stream);
}

long long jk_zmlp_features(int n, const double *dA, const int *J, int step, float *dX, double *dWg, void *stream)
{
  return features(1, n, dA, J, step, dX, dWg, stream);
}

int jk_mlp_forward(int nf, int count, const float *dX, const float *dParams, float *dY, void *stream)
{
  if (nf != kMlpFeat) return -1;
  if (count < 0) return -2;
  if (!count) return 0;
  Guard g;
  unsigned short *w = nullptr;
  float *b = nullptr;
  cudaStream_t s = (cudaStream_t)stream;
  CK(g.alloc(&w, (kMlpHidden * nf + kMlpHidden * kMlpHidden + kMlpHidden) * sizeof(unsigned short)));
  CK(g.alloc(&b, (2 * kMlpHidden + 1) * sizeof(float)));
  CK(mlp_pack(nf, dParams, w, b, s));
  CK(mlp_forward(nf, count, dX, w, b, dY, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

long long jk_mlp_grad_workspace(int nf, int count)
{
  if (nf != kMlpFeat || count <= 0) return -1;
  return (long long)mlp_grad_partial_floats(nf, count);
}

int jk_mlp_grad(int nf, int count, const float *dX, const float *dT, const float *dParams, float *dGrad, float *dLoss,
                float *dWork, void *stream)
{
  if (nf != kMlpFeat) return -1;
  if (count <= 0) return -2;
  if (!dX || !dT || !dParams || !dGrad || !dLoss || !dWork) return -3;
  CK(mlp_grad(nf, count, dX, dT, dParams, dGrad, dLoss, dWork, (cudaStream_t)stream));
  return 0;
}

int jk_mlp_adam(int np, float *dParams, const float *dGrad, float *dM, float *dV, int t, float lr, float beta1,
                float beta2, float eps, void *stream)
{
  if (np <= 0 || t < 1) return -1;
  CK(mlp_adam(np, dParams, dGrad, dM, dV, t, lr, beta1, beta2, eps, (cudaStream_t)stream));
  return 0;
}

long long jk_last_launch_count(void) { return g_launches; }

double jk_fp64_peak(void)
{
  if (pick_device(nullptr)) return -1.0;
  return fp64_peak();
}

int jk_max_order(int complex_) { return max_order(complex_ ? 1 : 0); }

const char *jk_strerror(int info)
{
  if (info >= 0) return "OK (number of steps)";
  switch (info) {
  case -1: return "N < 3";
  case -3: return "LDU < N";
  case -5: return "LDA < N";
  case -7: return "LDZ < N";
  case -8: return "J is NULL";
  case -16: return "N_2 < 0";
  case -10: return "a 2x2 hyperbolic transformation with |tanh| >= 1 (KHSVD2U)";
  case -11: return "a 2x2 hyperbolic transformation with |tanh| >= 1 (KHSVD2L)";
  case JK_ERR_ID_NCP: return "ID_NCP not in 0..3";
  case JK_ERR_ID_TRU: return "ID_TRU not in 0..2";
  case JK_ERR_J: return "a J entry is neither +1 nor -1";
  case JK_ERR_MAX_STEPS: return "the step limit was reached";
  case JK_ERR_CUDA: return "CUDA runtime error";
  case JK_ERR_NOMEM: return "device memory allocation failed";
  case JK_ERR_TOO_LARGE: return "N too large for this build";
  case JK_ERR_NO_DEVICE: return "no CUDA device";
  case JK_ERR_SCRATCH: return "N beyond the static scratch of jk_dweights_noalloc (JK_NOALLOC_MAX_N = 1024)";
  case JK_ERR_STALL: return "internal: the device loop neither advanced nor ended";
  case JK_ERR_STATE: return "a solver call out of order (or resume of a complex solve)";
  default: return "a 2x2 HSVD error (NaN or infinity in a pivot block) or argument error";
  }
}

}  // extern "C"
