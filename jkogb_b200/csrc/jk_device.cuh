// jk_device.cuh -- device helpers shared by the step-loop kernels (jk_kernels.cu)
// and the batched solver (jk_batch.cu): the real/complex scalar traits, the
// "may transform" test of the weight functions, the record-order keys and the
// 2x2 part of the hyperbolic pair weight.
#pragma once

#include "jk_math.cuh"
#include "jk_zmath.cuh"

namespace jk {

// ---------------------------------------------------------------------------
// scalar traits: the real (double) and complex (double2) flavours
// ---------------------------------------------------------------------------
template <typename T> struct Tr;

template <> struct Tr<double> {
  typedef Rot R;
  static __device__ __forceinline__ double zero() { return 0.0; }
  static __device__ __forceinline__ double one() { return 1.0; }
  static __device__ __forceinline__ double re(double a) { return a; }
  static __device__ __forceinline__ bool nonzero(double a) { return a != 0.0; }
  static __device__ __forceinline__ bool imnz(double) { return false; }
  static __device__ __forceinline__ double conj_(double a) { return a; }
  static __device__ __forceinline__ double neg_(double a) { return -a; }
  static __device__ __forceinline__ double magt(double aqp, double apq) { return dasum2(aqp, apq); }
  static __device__ __forceinline__ void hsvd2(double A[4], int j0, int j1, double U[4], double Z[4], double th1, int &info) { dhsvd2(A, j0, j1, U, Z, th1, info); }
  static __device__ __forceinline__ R ba(const double B[4], int) { return rot_ba(B); }
  static __device__ __forceinline__ R ab(const double B[4]) { return rot_ab(B); }
  static __device__ __forceinline__ void apply_ba(const R &t, double &x, double &y) { rot_apply(t, x, y); }
  static __device__ __forceinline__ void apply_ab(const R &t, double &x, double &y) { rot_apply(t, x, y); }
  // UT2, src/D/dtransf.F90:42-51
  static __device__ __forceinline__ void ut2(double V[4]) { const double t = V[M21]; V[M21] = V[M12]; V[M12] = t; }
};

template <> struct Tr<double2> {
  typedef ZRot R;
  static __device__ __forceinline__ double2 zero() { return make_double2(0.0, 0.0); }
  static __device__ __forceinline__ double2 one() { return make_double2(1.0, 0.0); }
  static __device__ __forceinline__ double re(double2 a) { return a.x; }
  static __device__ __forceinline__ bool nonzero(double2 a) { return !zeq0(a); }
  static __device__ __forceinline__ bool imnz(double2 a) { return a.y != 0.0; }
  static __device__ __forceinline__ double2 conj_(double2 a) { return conj(a); }
  static __device__ __forceinline__ double2 neg_(double2 a) { return zneg(a); }
  static __device__ __forceinline__ double magt(double2 aqp, double2 apq) { return dasum4(aqp.x, aqp.y, apq.x, apq.y); }
  static __device__ __forceinline__ void hsvd2(double2 A[4], int j0, int j1, double2 U[4], double2 Z[4], double th1, int &info) { zhsvd2(A, j0, j1, U, Z, th1, info); }
  static __device__ __forceinline__ R ba(const double2 B[4], int quirk) { return zrot_ba(B, quirk); }
  static __device__ __forceinline__ R ab(const double2 B[4]) { return zrot_ab(B); }
  static __device__ __forceinline__ void apply_ba(const R &t, double2 &x, double2 &y) { zrot_apply_ba(t, x, y); }
  static __device__ __forceinline__ void apply_ab(const R &t, double2 &x, double2 &y) { zrot_apply_ab(t, x, y); }
  // UH2, src/Z/ztransf.F90:79-90
  static __device__ __forceinline__ void ut2(double2 V[4])
  {
    V[M11] = conj(V[M11]);
    const double2 u21 = V[M21];
    V[M21] = conj(V[M12]);
    V[M12] = conj(u21);
    V[M22] = conj(V[M22]);
  }
};

__device__ __forceinline__ double nan_w() { return __longlong_as_double(0x7FF8000000000000LL); }

// "a transformation may be needed" of DMAGF2T/DMAGF2H (src/D/dstep.F90:19-20, 49-50)
// and ZMAGF2T/ZMAGF2H (src/Z/zstep.F90:19-21, 51-52)
template <typename T>
__device__ __forceinline__ bool may_transform(T app, T aqp, T apq, T aqq)
{
  return Tr<T>::nonzero(aqp) || Tr<T>::nonzero(apq) || Tr<T>::imnz(app) || Tr<T>::imnz(aqq) ||
         neg(Tr<T>::re(app)) || neg(Tr<T>::re(aqq));
}

// order-preserving 64-bit key of a weight; 0 for NaN (no record); -0 == +0
__device__ __forceinline__ unsigned long long wkey(double w)
{
  if (w != w) return 0ULL;
  const unsigned long long b = (unsigned long long)__double_as_longlong((w == 0.0) ? 0.0 : w);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
}

// the tie key: larger band first, then larger p (0-based indices, n <= 65535)
__device__ __forceinline__ unsigned tkey(int u, int v)
{
  const int p = (u < v) ? u : v, b = (u < v) ? (v - u) : (u - v);
  return ((unsigned)b << 16) | (unsigned)p;
}

__device__ __forceinline__ bool kbetter(unsigned long long k1, unsigned t1, unsigned long long k2, unsigned t2)
{
  return (k1 > k2) || ((k1 == k2) && (t1 > t2));
}

// The 2x2 part of DMAGF2H (src/D/dstep.F90:41-72) for the hyperbolic pair p < q with
// entries app, aqp, apq, aqq and J(p) = jp, J(q) = -jp.  Returns true when the pair
// needs the column scan of ABODNDF2 (then d holds its two leading terms and t the
// coefficients of Z2); otherwise w is the weight (NaN: no transformation).
__device__ __forceinline__ bool hyp_setup(double app, double aqp, double apq, double aqq, int jp, double &w, double &d, Rot &t)
{
  w = nan_w();
  if (!may_transform(app, aqp, apq, aqq)) return false;
  double A2[4] = { app, aqp, apq, aqq }, U2[4], Z2[4];
  int info = 0;
  dhsvd2(A2, jp, -jp, U2, Z2, JK_TH1FIX, info);
  if (info < 0) return false;
  if (!(info & 1)) { w = 0.0; return false; }
  if (!(info & 4)) { w = dasum2(aqp, apq); return false; }
  const double a1 = (info & 8) ? A2[M21] : 0.0, a2 = (info & 8) ? A2[M12] : 0.0;
  d = 0.0;
  d = fma(__dsub_rn(aqp, a1), __dadd_rn(aqp, a1), d);
  d = fma(__dsub_rn(apq, a2), __dadd_rn(apq, a2), d);
  t = rot_ab(Z2);
  return true;
}

// hyp_setup with the pair's 2x2 right transformation Z2 (column-major) instead of its AB
// coefficients, for the Gram form of the scanned weight
__device__ __forceinline__ bool hyp_setup_z(double app, double aqp, double apq, double aqq, int jp, double &w, double &d,
                                            double Z2[4])
{
  w = nan_w();
  if (!may_transform(app, aqp, apq, aqq)) return false;
  double A2[4] = { app, aqp, apq, aqq }, U2[4];
  int info = 0;
  dhsvd2(A2, jp, -jp, U2, Z2, JK_TH1FIX, info);
  if (info < 0) return false;
  if (!(info & 1)) { w = 0.0; return false; }
  if (!(info & 4)) { w = dasum2(aqp, apq); return false; }
  const double a1 = (info & 8) ? A2[M21] : 0.0, a2 = (info & 8) ? A2[M12] : 0.0;
  d = 0.0;
  d = fma(__dsub_rn(aqp, a1), __dadd_rn(aqp, a1), d);
  d = fma(__dsub_rn(apq, a2), __dadd_rn(apq, a2), d);
  return true;
}

// the Gram form of a scanned hyperbolic weight: d + nx (1 - Z11^2 - Z12^2) +
// ny (1 - Z21^2 - Z22^2) - 2 (Z11 Z21 + Z12 Z22) g, with nx, ny, g the squared norms and the
// product of the pair's columns without rows p, q (the terms 1 - Z11^2 - Z12^2 and
// 1 - Z21^2 - Z22^2 formed without cancellation at Z11, Z22 near +-1)
__device__ __forceinline__ double gram_weight(double d, const double Z2[4], double nx, double ny, double g)
{
  const double z11 = Z2[M11], z21 = Z2[M21], z12 = Z2[M12], z22 = Z2[M22];
  const double c1 = (1.0 - z11) * (1.0 + z11) - z12 * z12;
  const double c2 = (1.0 - z22) * (1.0 + z22) - z21 * z21;
  const double c3 = z11 * z21 + z12 * z22;
  return d + (nx * c1 + ny * c2 - 2.0 * c3 * g);
}

}  // namespace jk
