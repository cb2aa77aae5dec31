"""jkogb_b200: the J-Kogbetliantz hyperbolic SVD step loop of venovako/JKogb on a B200.

Python host side of libjkogb_b200.so (C ABI in include/jkogb.h).  It mirrors the
reference's interface for this path:

  dstep_loop / zstep_loop   DSTEP_LOOP / ZSTEP_LOOP (src/D/dstep.F90:472, src/Z/zstep.F90:482)
  step_loop                 either, chosen by the dtype of Y
  step_loop_dev             the same on torch CUDA tensors, on the current stream
  hsvd2_batch               DHSVD2 / ZHSVD2 on a batch of 2x2 blocks (src/D/dtransf.F90:614)
  weights                   one build's pair weights (DMAGF2T/H, src/D/dstep.F90:12-72)
  select                    the greedy non-colliding selection (AW_NCP1/2, src/shared/atypes.F90:359-484)
  read_yj / write_uzs       the FN.Y / FN.J -> FN.YU / FN.ZZ / FN.SY file contract (src/D/bio.F90)

All compute runs in the CUDA library; there is no CPU fallback.  Importing this
module does not need a GPU, calling the compute entry points does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

__all__ = ["lib", "step_loop", "dstep_loop", "zstep_loop", "step_loop_dev", "hsvd2_batch", "weights", "select",
           "read_yj", "write_uzs", "JkError", "jstep_len", "SYMBOLS", "weights_noalloc",
           "NOALLOC_MAX_N", "dstep_loop_batched", "Batch", "batch_pack", "batch_unpack", "BATCH_MAX_N", "Solver"]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libjkogb_b200.so")

# every symbol include/jkogb.h declares
SYMBOLS = ("jk_dstep_loop", "jk_zstep_loop", "jk_dstep_loop_dev", "jk_zstep_loop_dev", "jk_solver_create",
           "jk_solver_destroy", "jk_solver_begin", "jk_solver_resume", "jk_solver_advance", "jk_solver_steps",
           "jk_solver_finish", "jk_dhsvd2_batch",
           "jk_zhsvd2_batch", "jk_dweights", "jk_zweights", "jk_select", "jk_handle_create", "jk_handle_destroy",
           "jk_handle_weights", "jk_dweights_noalloc", "jk_batch_create", "jk_batch_destroy",
           "jk_batch_run", "jk_batch_tune", "jk_batch_set_scorer", "jk_dstep_loop_batched", "jk_mlp_nparams", "jk_scorer_create",
           "jk_scorer_destroy", "jk_dstep_loop_dev_scored", "jk_zstep_loop_dev_scored", "jk_mlp_features",
           "jk_zmlp_features", "jk_mlp_forward", "jk_mlp_grad_workspace",
           "jk_mlp_grad", "jk_mlp_adam", "jk_last_launch_count", "jk_fp64_peak", "jk_max_order", "jk_strerror")


class JkError(RuntimeError):
    """A negative INFO from the library (or a missing library)."""

    def __init__(self, info: int, what: str = ""):
        self.info = info
        super().__init__(f"{what}INFO={info}: {strerror(info) if _lib is not None else ''}")


class Opts(C.Structure):
    _fields_ = [("max_steps", C.c_int), ("zba_quirk", C.c_int), ("graph_steps", C.c_int), ("device", C.c_int),
                ("reserved", C.c_int * 4)]


class Trace(C.Structure):
    _fields_ = [("max_steps", C.c_int), ("sl", C.POINTER(C.c_int)), ("nl", C.POINTER(C.c_int)),
                ("trig", C.POINTER(C.c_int)), ("hyp", C.POINTER(C.c_int)), ("tw", C.POINTER(C.c_double)),
                ("rounds", C.POINTER(C.c_int)), ("max_piv", C.c_longlong), ("piv", C.POINTER(C.c_int)),
                ("n_piv", C.c_longlong), ("n_steps", C.c_int)]


_lib = None


def lib():
    """Load libjkogb_b200.so (built in-tree by build()); raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise JkError(-30, f"libjkogb_b200.so not built ({LIB_PATH}); run jkogb_b200.build.build(): ")
        L = C.CDLL(LIB_PATH)
        dp, ip, vp = C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_void_p
        for nm in ("jk_dstep_loop", "jk_zstep_loop"):
            f = getattr(L, nm)
            f.restype = C.c_int
            f.argtypes = [C.c_int, vp, C.c_int, vp, C.c_int, vp, C.c_int, ip, vp, C.c_int, C.c_int, C.c_int,
                          C.POINTER(Opts), C.POINTER(Trace)]
        for nm in ("jk_dstep_loop_dev", "jk_zstep_loop_dev"):
            f = getattr(L, nm)
            f.restype = C.c_int
            f.argtypes = [C.c_int, vp, vp, vp, ip, vp, C.c_int, C.c_int, C.c_int, C.POINTER(Opts), C.POINTER(Trace), vp]
        L.jk_solver_create.restype = C.c_void_p
        L.jk_solver_create.argtypes = [C.c_int, C.c_int, ip, C.c_int, C.c_int, C.c_int, C.POINTER(Opts), ip]
        L.jk_solver_destroy.restype = None
        L.jk_solver_destroy.argtypes = [C.c_void_p]
        L.jk_solver_begin.restype = C.c_int
        L.jk_solver_begin.argtypes = [C.c_void_p, vp, vp, vp, vp]
        L.jk_solver_resume.restype = C.c_int
        L.jk_solver_resume.argtypes = [C.c_void_p, vp, vp, vp, vp, C.c_longlong, vp]
        L.jk_solver_advance.restype = C.c_int
        L.jk_solver_advance.argtypes = [C.c_void_p, C.c_longlong]
        L.jk_solver_steps.restype = C.c_longlong
        L.jk_solver_steps.argtypes = [C.c_void_p]
        L.jk_solver_finish.restype = C.c_int
        L.jk_solver_finish.argtypes = [C.c_void_p, vp]
        for nm in ("jk_dhsvd2_batch", "jk_zhsvd2_batch"):
            f = getattr(L, nm)
            f.restype = C.c_int
            f.argtypes = [C.c_int, vp, ip, vp, vp, ip, C.c_double]
        for nm in ("jk_dweights", "jk_zweights"):
            f = getattr(L, nm)
            f.restype = C.c_int
            f.argtypes = [C.c_int, vp, C.c_int, ip, dp]
        L.jk_select.restype = C.c_int
        L.jk_select.argtypes = [C.c_int, dp, C.c_int, ip]
        L.jk_handle_create.restype = C.c_void_p
        L.jk_handle_create.argtypes = [C.c_int, C.c_int, ip, ip]
        L.jk_handle_destroy.restype = None
        L.jk_handle_destroy.argtypes = [C.c_void_p]
        L.jk_handle_weights.restype = C.c_int
        L.jk_handle_weights.argtypes = [C.c_void_p, vp, vp, vp]
        L.jk_dweights_noalloc.restype = C.c_int
        L.jk_dweights_noalloc.argtypes = [C.c_int, vp, ip, vp, vp]
        L.jk_batch_create.restype = C.c_void_p
        L.jk_batch_create.argtypes = [C.c_int, ip, ip, ip, C.POINTER(Opts), ip]
        L.jk_batch_destroy.restype = None
        L.jk_batch_destroy.argtypes = [C.c_void_p]
        L.jk_batch_run.restype = C.c_int
        L.jk_batch_run.argtypes = [C.c_void_p, vp, vp, vp, vp, vp, vp]
        L.jk_batch_tune.restype = C.c_int
        L.jk_batch_tune.argtypes = [C.c_void_p, vp, vp, vp, vp, vp, vp]
        L.jk_batch_set_scorer.restype = C.c_int
        L.jk_batch_set_scorer.argtypes = [C.c_void_p, C.c_void_p]
        L.jk_mlp_nparams.restype = C.c_int
        L.jk_mlp_nparams.argtypes = [C.c_int]
        L.jk_scorer_create.restype = C.c_void_p
        L.jk_scorer_create.argtypes = [C.c_int, C.POINTER(C.c_float), C.c_int, ip]
        L.jk_scorer_destroy.restype = None
        L.jk_scorer_destroy.argtypes = [C.c_void_p]
        for nm in ("jk_dstep_loop_dev_scored", "jk_zstep_loop_dev_scored"):
            getattr(L, nm).restype = C.c_int
            getattr(L, nm).argtypes = [C.c_int, vp, vp, vp, ip, vp, C.c_int, C.c_void_p, C.POINTER(Opts),
                                       C.POINTER(Trace), ip, vp]
        for nm in ("jk_mlp_features", "jk_zmlp_features"):
            getattr(L, nm).restype = C.c_longlong
            getattr(L, nm).argtypes = [C.c_int, vp, ip, C.c_int, vp, vp, vp]
        L.jk_mlp_forward.restype = C.c_int
        L.jk_mlp_forward.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp]
        L.jk_mlp_grad_workspace.restype = C.c_longlong
        L.jk_mlp_grad_workspace.argtypes = [C.c_int, C.c_int]
        L.jk_mlp_grad.restype = C.c_int
        L.jk_mlp_grad.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp]
        L.jk_mlp_adam.restype = C.c_int
        L.jk_mlp_adam.argtypes = [C.c_int, vp, vp, vp, vp, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, vp]
        L.jk_dstep_loop_batched.restype = C.c_int
        L.jk_dstep_loop_batched.argtypes = [C.c_int, ip, ip, vp, vp, vp, ip, vp, ip, C.POINTER(Opts)]
        L.jk_last_launch_count.restype = C.c_longlong
        L.jk_last_launch_count.argtypes = []
        L.jk_fp64_peak.restype = C.c_double
        L.jk_fp64_peak.argtypes = []
        L.jk_max_order.restype = C.c_int
        L.jk_max_order.argtypes = [C.c_int]
        L.jk_strerror.restype = C.c_char_p
        L.jk_strerror.argtypes = [C.c_int]
        _lib = L
    return _lib


def strerror(info: int) -> str:
    return lib().jk_strerror(int(info)).decode()


def jstep_len(n: int, n_2: int) -> int:
    """JSTEP_LEN, src/shared/jstep.F90:124-133."""
    if n_2 == 0:
        return max(n // 2, 0)
    return min(max(n_2, 0), n // 2)


def _opts(max_steps=0, zba_quirk=0, graph_steps=0, device=0):
    o = Opts()
    o.max_steps, o.zba_quirk, o.graph_steps, o.device = int(max_steps), int(zba_quirk), int(graph_steps), int(device)
    return o


def _new_trace(max_steps, max_piv):
    tr = Trace()
    bufs = dict(sl=np.zeros(max_steps, np.int32), nl=np.zeros(max_steps, np.int32), trig=np.zeros(max_steps, np.int32),
                hyp=np.zeros(max_steps, np.int32), tw=np.zeros(max_steps, np.float64),
                rounds=np.zeros(max_steps, np.int32), piv=np.zeros(2 * max_piv, np.int32))
    tr.max_steps, tr.max_piv = max_steps, max_piv
    for k in ("sl", "nl", "trig", "hyp", "rounds", "piv"):
        setattr(tr, k, bufs[k].ctypes.data_as(C.POINTER(C.c_int)))
    tr.tw = bufs["tw"].ctypes.data_as(C.POINTER(C.c_double))
    return tr, bufs


def _collect(tr, bufs):
    m = min(tr.n_steps, len(bufs["sl"]))
    return dict(n_steps=tr.n_steps, sl=bufs["sl"][:m].copy(), nl=bufs["nl"][:m].copy(), trig=bufs["trig"][:m].copy(),
                hyp=bufs["hyp"][:m].copy(), tw=bufs["tw"][:m].copy(), rounds=bufs["rounds"][:m].copy(),
                piv=bufs["piv"][:2 * tr.n_piv].reshape(-1, 2).copy())


def step_loop(Y, J, n_2=0, id_ncp=0, id_tru=0, trace=False, max_steps=0, zba_quirk=0, graph_steps=0,
              trace_steps=1 << 16, trace_piv=1 << 22):
    """DSTEP_LOOP / ZSTEP_LOOP on host arrays.  Y (n x n, float64 or complex128) is not modified.

    Returns dict(info, A, U, Z, sigma[, trace]) with A the final matrix (diagonal zeroed),
    U, Z such that Y = U diag(sigma) Z; raises JkError when INFO < 0.
    """
    Y = np.asarray(Y)
    n = Y.shape[0]
    cplx = np.iscomplexobj(Y)
    dt = np.complex128 if cplx else np.float64
    A = np.asfortranarray(Y.astype(dt, copy=True))
    U = np.empty((n, n), dt, order="F")
    Z = np.empty((n, n), dt, order="F")
    s = np.empty(n, np.float64)
    Jc = np.ascontiguousarray(np.asarray(J).astype(np.int32))
    o = _opts(max_steps, zba_quirk, graph_steps)
    trp, bufs = (_new_trace(trace_steps, trace_piv) if trace else (None, None))
    f = lib().jk_zstep_loop if cplx else lib().jk_dstep_loop
    info = f(n, U.ctypes.data, n, A.ctypes.data, n, Z.ctypes.data, n, Jc.ctypes.data_as(C.POINTER(C.c_int)),
             s.ctypes.data, int(n_2), int(id_ncp), int(id_tru), C.byref(o), C.byref(trp) if trace else None)
    if info < 0 and info != -24:
        raise JkError(info, "step loop: ")
    out = dict(info=info, A=A, U=U, Z=Z, sigma=s)
    if trace:
        out["trace"] = _collect(trp, bufs)
    return out


def dstep_loop(Y, J, n_2=0, id_ncp=0, id_tru=0, **kw):
    return step_loop(np.asarray(Y, np.float64), J, n_2, id_ncp, id_tru, **kw)


def zstep_loop(Y, J, n_2=0, id_ncp=0, id_tru=0, **kw):
    return step_loop(np.asarray(Y, np.complex128), J, n_2, id_ncp, id_tru, **kw)


def step_loop_dev(A, U, Z, sigma, J, n_2=0, id_ncp=0, id_tru=0, stream=None, max_steps=0, zba_quirk=0, graph_steps=0):
    """The loop on torch CUDA tensors (n x n, column-major, i.e. the transpose of a
    contiguous row-major tensor, float64 or complex128); J a host sequence.  A is
    overwritten, U, Z, sigma are outputs.  Returns INFO; raises JkError when INFO < 0."""
    import torch
    n = A.shape[0]
    cplx = A.dtype == torch.complex128
    for t in (A, U, Z):
        assert t.is_cuda and t.dtype == A.dtype and t.shape == (n, n)
        assert t.stride() == (1, n), "column-major n x n tensors are expected (e.g. X.t() of a contiguous tensor)"
    assert sigma.is_cuda and sigma.dtype == torch.float64 and sigma.numel() == n
    Jc = np.ascontiguousarray(np.asarray(J).astype(np.int32))
    o = _opts(max_steps, zba_quirk, graph_steps, A.device.index or 0)
    st = stream if stream is not None else torch.cuda.current_stream(A.device)
    f = lib().jk_zstep_loop_dev if cplx else lib().jk_dstep_loop_dev
    info = f(n, U.data_ptr(), A.data_ptr(), Z.data_ptr(), Jc.ctypes.data_as(C.POINTER(C.c_int)), sigma.data_ptr(),
             int(n_2), int(id_ncp), int(id_tru), C.byref(o), None, C.c_void_p(st.cuda_stream))
    if info < 0 and info != -24:
        raise JkError(info, "device step loop: ")
    return info


class Solver:
    """The step loop as a reusable object (jk_solver_*): one workspace for an order n, sign
    vector J, N_2 and strategy, advanced a given number of steps at a time on device
    buffers.  Pointers are raw device addresses (e.g. tensor.data_ptr()) of column-major
    n x n buffers; `stream` is a raw cudaStream_t."""

    def __init__(self, n, J, n_2=0, complex_=False, id_ncp=0, id_tru=0, max_steps=0, zba_quirk=0, graph_steps=0):
        Jc = np.ascontiguousarray(np.asarray(J).astype(np.int32))
        info = C.c_int(0)
        self.n = int(n)
        o = _opts(max_steps, zba_quirk, graph_steps)
        self._s = lib().jk_solver_create(self.n, int(bool(complex_)), Jc.ctypes.data_as(C.POINTER(C.c_int)), int(n_2),
                                          int(id_ncp), int(id_tru), C.byref(o), C.byref(info))
        if not self._s:
            raise JkError(info.value, "solver: ")

    def begin(self, dU, dA, dZ, stream=0):
        """Start a solve: A (in/out) is the input matrix, U = Z = I."""
        rc = lib().jk_solver_begin(self._s, C.c_void_p(dU), C.c_void_p(dA), C.c_void_p(dZ), C.c_void_p(stream))
        if rc < 0:
            raise JkError(rc, "solver begin: ")

    def resume(self, dU, dA, dZ, dsigma, steps, stream=0):
        """Continue a real loop that stopped after `steps` steps (A, U, Z, SIGMA as it left them)."""
        rc = lib().jk_solver_resume(self._s, C.c_void_p(dU), C.c_void_p(dA), C.c_void_p(dZ), C.c_void_p(dsigma),
                                    int(steps), C.c_void_p(stream))
        if rc < 0:
            raise JkError(rc, "solver resume: ")

    def advance(self, steps=0):
        """Run until S has grown by `steps` (0: to the end); True once the loop has ended."""
        rc = lib().jk_solver_advance(self._s, int(steps))
        if rc < 0:
            raise JkError(rc, "solver advance: ")
        return rc == 1

    @property
    def steps(self):
        return int(lib().jk_solver_steps(self._s))

    def finish(self, dsigma):
        """SIGMA, the zeroed diagonal, J Z^T J; returns INFO (JK_ERR_MAX_STEPS if not ended)."""
        info = lib().jk_solver_finish(self._s, C.c_void_p(dsigma))
        if info < 0 and info != -24:
            raise JkError(info, "solver finish: ")
        return info

    def close(self):
        if self._s:
            lib().jk_solver_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def hsvd2_batch(B, J, th1=0.75):
    """A batch of 2x2 HSVDs (DHSVD2 / ZHSVD2) on the GPU.  B: (count, 2, 2), J: (count, 2).
    Returns (A, U, Z, info) as DHSVD2 leaves them."""
    B = np.asarray(B)
    cplx = np.iscomplexobj(B)
    dt = np.complex128 if cplx else np.float64
    cnt = B.shape[0]
    A = np.ascontiguousarray(np.transpose(B.astype(dt), (0, 2, 1)))  # column-major 2x2 blocks
    U = np.empty_like(A)
    Z = np.empty_like(A)
    info = np.zeros(cnt, np.int32)
    Jc = np.ascontiguousarray(np.asarray(J, np.int32))
    f = lib().jk_zhsvd2_batch if cplx else lib().jk_dhsvd2_batch
    rc = f(cnt, A.ctypes.data, Jc.ctypes.data_as(C.POINTER(C.c_int)), U.ctypes.data, Z.ctypes.data,
           info.ctypes.data_as(C.POINTER(C.c_int)), float(th1))
    if rc < 0:
        raise JkError(rc, "hsvd2_batch: ")
    tr = lambda X: np.transpose(X, (0, 2, 1))  # noqa: E731
    return tr(A), tr(U), tr(Z), info


def weights(A, J):
    """Pair weights of one build on the GPU, as a symmetric n x n matrix (NaN = no transformation)."""
    A = np.asarray(A)
    n = A.shape[0]
    cplx = np.iscomplexobj(A)
    Af = np.asfortranarray(A.astype(np.complex128 if cplx else np.float64))
    W = np.empty((n, n), np.float64, order="F")
    Jc = np.ascontiguousarray(np.asarray(J, np.int32))
    f = lib().jk_zweights if cplx else lib().jk_dweights
    rc = f(n, Af.ctypes.data, n, Jc.ctypes.data_as(C.POINTER(C.c_int)), W.ctypes.data_as(C.POINTER(C.c_double)))
    if rc < 0:
        raise JkError(rc, "weights: ")
    return W


class Handle:
    """A device workspace for one order n and sign vector J (kernel-level entry points)."""

    def __init__(self, n, J, complex_=False):
        Jc = np.ascontiguousarray(np.asarray(J, np.int32))
        info = C.c_int(0)
        self.n = int(n)
        self._h = lib().jk_handle_create(self.n, int(bool(complex_)), Jc.ctypes.data_as(C.POINTER(C.c_int)),
                                          C.byref(info))
        if not self._h:
            raise JkError(info.value, "handle: ")

    def weights(self, dA_ptr, dW_ptr=None, stream=0):
        """Enqueue one build's weights of the device matrix at dA_ptr on `stream` (a raw cudaStream_t)."""
        rc = lib().jk_handle_weights(self._h, C.c_void_p(dA_ptr), C.c_void_p(dW_ptr or 0), C.c_void_p(stream))
        if rc < 0:
            raise JkError(rc, "handle weights: ")

    def close(self):
        if self._h:
            lib().jk_handle_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


NOALLOC_MAX_N = 1024  # JK_NOALLOC_MAX_N


def weights_noalloc(n, dA_ptr, J, dW_ptr, stream=0):
    """jk_dweights_noalloc: the weights of the real device matrix at dA_ptr (n x n, column-major)
    into the device matrix at dW_ptr (off-diagonal entries), enqueued on `stream` (a raw
    cudaStream_t), with no device allocation; all calls on a device share one static scratch."""
    Jc = np.ascontiguousarray(np.asarray(J, np.int32))
    if Jc.shape != (int(n),):
        raise ValueError("J must hold n signs")
    rc = lib().jk_dweights_noalloc(int(n), C.c_void_p(dA_ptr), Jc.ctypes.data_as(C.POINTER(C.c_int)),
                                   C.c_void_p(dW_ptr), C.c_void_p(stream))
    if rc < 0:
        raise JkError(rc, "weights_noalloc: ")


BATCH_MAX_N = 128  # JK_BATCH_MAX_N


def batch_pack(mats, Js):
    """Pack real square matrices (column-major blocks, one after the other) and their sign
    vectors the way the batched entry points expect; returns (A, J, n, offsets)."""
    n = np.array([np.asarray(Y).shape[0] for Y in mats], np.int32)
    off = np.concatenate([[0], np.cumsum(n.astype(np.int64) ** 2)])
    A = np.empty(int(off[-1]), np.float64)
    for m, Y in enumerate(mats):
        A[off[m]:off[m + 1]] = np.asarray(Y, np.float64).ravel(order="F")
    J = np.ascontiguousarray(np.concatenate([np.asarray(j) for j in Js]).astype(np.int32))
    return A, J, n, off


def batch_unpack(X, n, off):
    """The column-major blocks of a packed batch as a list of n x n arrays."""
    return [X[off[m]:off[m + 1]].reshape((n[m], n[m]), order="F") for m in range(len(n))]


def dstep_loop_batched(mats, Js, n_2=None, max_steps=0):
    """jk_dstep_loop_batched on host arrays: every matrix through the whole step loop in one
    persistent launch.  n_2: per-matrix N_2 (default 0, i.e. N/2).  Returns a list of dicts
    (info, A, U, Z, sigma) as dstep_loop returns them."""
    A, J, n, off = batch_pack(mats, Js)
    cnt = len(n)
    n2 = np.ascontiguousarray(np.zeros(cnt, np.int32) if n_2 is None else np.asarray(n_2, np.int32))
    U = np.empty_like(A)
    Z = np.empty_like(A)
    sig = np.empty(int(np.sum(n)), np.float64)
    info = np.zeros(cnt, np.int32)
    o = _opts(max_steps)
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))  # noqa: E731
    rc = lib().jk_dstep_loop_batched(cnt, ip(n), ip(n2), A.ctypes.data, U.ctypes.data, Z.ctypes.data, ip(J),
                                     sig.ctypes.data, ip(info), C.byref(o))
    if rc < 0:
        raise JkError(rc, "batched step loop: ")
    so = np.concatenate([[0], np.cumsum(n)])
    As, Us, Zs = batch_unpack(A, n, off), batch_unpack(U, n, off), batch_unpack(Z, n, off)
    return [dict(info=int(info[m]), A=As[m], U=Us[m], Z=Zs[m], sigma=sig[so[m]:so[m + 1]]) for m in range(cnt)]


class Batch:
    """A plan of the batched solver for one batch shape (jk_batch_create); run() and tune()
    take raw device pointers of the packed buffers (see batch_pack)."""

    def __init__(self, n, n_2, J, max_steps=0):
        self.n = np.ascontiguousarray(np.asarray(n, np.int32))
        self.n_2 = np.ascontiguousarray(np.asarray(n_2, np.int32))
        Jc = np.ascontiguousarray(np.asarray(J, np.int32))
        info = C.c_int(0)
        o = _opts(max_steps)
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))  # noqa: E731
        self._b = lib().jk_batch_create(len(self.n), ip(self.n), ip(self.n_2), ip(Jc), C.byref(o), C.byref(info))
        if not self._b:
            raise JkError(info.value, "batch plan: ")

    def run(self, dA, dU, dZ, dsigma, dinfo, stream=0):
        rc = lib().jk_batch_run(self._b, dA, dU, dZ, dsigma, dinfo, C.c_void_p(stream))
        if rc < 0:
            raise JkError(rc, "batch run: ")

    def set_scorer(self, scorer):
        """Rank by the Gram form of the scanned weights (a scorer.Scorer made without a
        network), or by the exact weights (None)."""
        rc = lib().jk_batch_set_scorer(self._b, scorer._s if scorer is not None else None)
        if rc < 0:
            raise JkError(rc, "batch scorer: ")

    def tune(self, dA, dU, dZ, dsigma, dinfo, stream=0):
        """Choose the block shape on this batch; returns the chosen threads per block."""
        rc = lib().jk_batch_tune(self._b, dA, dU, dZ, dsigma, dinfo, C.c_void_p(stream))
        if rc < 0:
            raise JkError(rc, "batch tune: ")
        return rc

    def close(self):
        if self._b:
            lib().jk_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def select(W, n_2):
    """The greedy non-colliding selection on the GPU from a symmetric n x n weight matrix;
    returns the (SL, 2) pivots (1-based p < q) in selection order."""
    W = np.asfortranarray(np.asarray(W, np.float64))
    n = W.shape[0]
    piv = np.zeros(2 * max(n // 2, 1), np.int32)
    sl = lib().jk_select(n, W.ctypes.data_as(C.POINTER(C.c_double)), int(n_2), piv.ctypes.data_as(C.POINTER(C.c_int)))
    if sl < 0:
        raise JkError(sl, "select: ")
    return piv[:2 * sl].reshape(-1, 2).copy()


# ---- the file contract of djk / zjk (README.md:53-57; src/shared/binio.F90, src/D/bio.F90) ----

def read_yj(fn: str, n: int, complex_: bool = False):
    """Read FN.Y (n x n column-major float64 / complex128) and FN.J (n int64)."""
    dt = np.complex128 if complex_ else np.float64
    y = np.fromfile(fn + ".Y", dtype=dt, count=n * n)
    if y.size != n * n:
        raise JkError(1, f"{fn}.Y holds {y.size} of {n * n} entries: ")
    j = np.fromfile(fn + ".J", dtype=np.int64, count=n)
    if j.size != n:
        raise JkError(2, f"{fn}.J holds {j.size} of {n} entries: ")
    return y.reshape((n, n), order="F"), j


def write_uzs(fn: str, U, Z, S):
    """Write FN.YU, FN.ZZ (n x n column-major) and FN.SY (n float64)."""
    np.asfortranarray(U).ravel(order="F").tofile(fn + ".YU")
    np.asfortranarray(Z).ravel(order="F").tofile(fn + ".ZZ")
    np.asarray(S, np.float64).tofile(fn + ".SY")


def write_yj(fn: str, Y, J):
    """Write FN.Y and FN.J (the inputs djk / zjk read)."""
    np.asfortranarray(Y).ravel(order="F").tofile(fn + ".Y")
    np.asarray(J, np.int64).tofile(fn + ".J")
