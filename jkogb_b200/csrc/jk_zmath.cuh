// jk_zmath.cuh -- device complex 2x2 HSVD of the J-Kogbetliantz step
// (src/Z/ztransf.F90), operation for operation; complex values are double2.
#pragma once

#include "jk_math.cuh"

namespace jk {

__device__ __forceinline__ void zswap(double2 &a, double2 &b) { const double2 t = a; a = b; b = t; }

// C1A, src/Z/ztransf.F90:231-241
__device__ __forceinline__ void zc1a(const double B[4], double2 &a1, double2 &a2)
{
  const double2 c1 = zddiv(zdfma(B[M12], a2, a1), B[M11]);
  const double2 c2 = zddiv(zdfma(B[M21], a1, a2), B[M22]);
  a1 = c1; a2 = c2;
}

// C2A, src/Z/ztransf.F90:245-258
__device__ __forceinline__ void zc2a(const double B[4], double2 A[4])
{
  double2 C[4];
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    C[2 * j + 0] = zddiv(zdfma(B[M12], A[2 * j + 1], A[2 * j + 0]), B[M11]);
    C[2 * j + 1] = zddiv(zdfma(B[M21], A[2 * j + 0], A[2 * j + 1]), B[M22]);
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) A[k] = C[k];
}

// A2C, src/Z/ztransf.F90:262-275
__device__ __forceinline__ void za2c(double2 A[4], const double B[4])
{
  double2 C[4];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    C[i + 0] = zddiv(zdfma(B[M21], A[i + 2], A[i + 0]), B[M11]);
    C[i + 2] = zddiv(zdfma(B[M12], A[i + 0], A[i + 2]), B[M22]);
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) A[k] = C[k];
}

// ZPOLAR, src/Z/ztransf.F90:112-126
__device__ __forceinline__ void zpolar(double2 z, double &a, double2 &e)
{
  a = hypot2(z.x, z.y);
  const double c = copysign(fmin(__ddiv_rn(fabs(z.x), a), 1.0), z.x);
  const double s = __ddiv_rn(z.y, fmax(a, JK_MINF));
  e = zc(c, s);
}

// ZHSVD2T, src/Z/ztransf.F90:641-835
__device__ __forceinline__ void zhsvd2t(double2 A[4], const int J0, const int J1, double2 U[4], double2 Z[4], int &info)
{
  double c, t, w;
  double2 r, s;
  bool p, d = true;
  if (zeq0(A[M21])) c = zabs(A[M11]);
  else if (zeq0(A[M11])) { c = zabs(A[M21]); d = false; }
  else { c = hypot2(zabs(A[M11]), zabs(A[M21])); d = false; }
  if (zeq0(A[M12])) t = zabs(A[M22]);
  else if (zeq0(A[M22])) { t = zabs(A[M12]); d = false; }
  else { t = hypot2(zabs(A[M12]), zabs(A[M22])); d = false; }

  if (c < t) {
    zswap(A[M11], A[M12]); zswap(A[M21], A[M22]);
    if (J0 == J1) { zswap(Z[M11], Z[M12]); zswap(Z[M21], Z[M22]); }
    p = true;
    w = t;
  }
  else { p = false; w = c; }

  zpolar(A[M11], c, r);
  if (zne1(r)) {
    s = conj(r);
    U[M11] = zzmul(U[M11], s); U[M12] = zzmul(U[M12], s);
    A[M11] = zzmul(A[M11], s); A[M12] = zzmul(A[M12], s);
  }
  zpolar(A[M21], t, s);
  if (zne1(s)) {
    r = conj(s);
    U[M21] = zzmul(U[M21], r); U[M22] = zzmul(U[M22], r);
    A[M21] = zzmul(A[M21], r); A[M22] = zzmul(A[M22], r);
  }

  if (A[M11].x < A[M21].x) {
    zswap(U[M11], U[M21]); zswap(U[M12], U[M22]);
    zswap(A[M11], A[M21]); zswap(A[M12], A[M22]);
  }

  if (!d) {
    t = __ddiv_rn(A[M21].x, A[M11].x);
    c = sqrt(fma(t, t, 1.0));
    const double Q[4] = { c, -t, t, c };
    zc2a(Q, U);
    zc1a(Q, A[M12], A[M22]);
  }
  A[M11] = zc(w, 0.0);
  A[M21] = zc(0.0, 0.0);

  if ((J0 != J1) && p) {
    zswap(A[M11], A[M12]); zswap(A[M21], A[M22]);
    zswap(U[M11], U[M21]); zswap(U[M12], U[M22]);
    zswap(A[M11], A[M21]); zswap(A[M12], A[M22]);
    zpolar(A[M21], t, s);
    if (zne1(s)) {
      r = conj(s);
      Z[M11] = zzmul(Z[M11], r); Z[M21] = zzmul(Z[M21], r);
      A[M11] = zzmul(A[M11], r); A[M21] = zzmul(A[M21], r);
    }
    zpolar(A[M11], c, r);
    if (zne1(r)) {
      s = conj(r);
      U[M11] = zzmul(U[M11], s); U[M12] = zzmul(U[M12], s);
      A[M11] = zzmul(A[M11], s);
    }
  }
  else {
    zpolar(A[M12], c, r);
    if (zne1(r)) {
      s = conj(r);
      Z[M12] = zzmul(Z[M12], s); Z[M22] = zzmul(Z[M22], s);
      A[M12] = zzmul(A[M12], s); A[M22] = zzmul(A[M22], s);
    }
    zpolar(A[M22], t, s);
    if (zne1(s)) {
      r = conj(s);
      U[M21] = zzmul(U[M21], r); U[M22] = zzmul(U[M22], r);
      A[M22] = zzmul(A[M22], r);
    }
  }
  info = d ? 0 : 1;
}

// ZHSVD2S, src/Z/ztransf.F90:839-880
__device__ __forceinline__ void zhsvd2s(double2 A[4], const int J0, const int J1, double2 U[4], double2 Z[4], int &info)
{
  const int t = J0 + J1;
  if (((t == 2) && (A[M11].x < A[M22].x)) || ((t == -2) && (A[M22].x < A[M11].x))) {
    A[M21] = U[M11]; A[M12] = U[M12];
    U[M11] = U[M21]; U[M12] = U[M22];
    U[M21] = A[M21]; U[M22] = A[M12];
    A[M21] = A[M11]; A[M11] = A[M22]; A[M22] = A[M21];
    A[M21] = Z[M11]; A[M12] = Z[M21];
    Z[M11] = Z[M12]; Z[M21] = Z[M22];
    Z[M12] = A[M21]; Z[M22] = A[M12];
  }
  if (!(info & 8)) { A[M21] = zc(0.0, 0.0); A[M12] = zc(0.0, 0.0); }
  if (zne1(U[M11]) || !zeq0(U[M21]) || !zeq0(U[M12]) || zne1(U[M22])) info += 2;
  if (zne1(Z[M11]) || !zeq0(Z[M21]) || !zeq0(Z[M12]) || zne1(Z[M22])) info += 4;
}

// ZSCALEA, src/Z/ztransf.F90:884-921
__device__ __forceinline__ void zscalea(double2 A[4], int &s)
{
  s = 0x7FFFFFFF;
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      double aa = fabs(A[2 * j + i].x);
      if (!(aa <= JK_HUGE)) { s = -((j + 1) * 2 + (i + 1)); return; }
      s = imin(s, JK_EH - exponent(fmax(aa, JK_MINF)) - 2);
      aa = fabs(A[2 * j + i].y);
      if (!(aa <= JK_HUGE)) { s = -((j + 1) * 2 + (i + 1)); return; }
      s = imin(s, JK_EH - exponent(fmax(aa, JK_MINF)) - 2);
    }
  if (s != 0)
#pragma unroll
    for (int k = 0; k < 4; ++k) A[k] = zc(scale(A[k].x, s), scale(A[k].y, s));
}

// ZHSVD2 (argument-checking form), src/Z/ztransf.F90:925-1009
__device__ __forceinline__ void zhsvd2(double2 A[4], const int J0, const int J1, double2 U[4], double2 Z[4], double th1, int &info)
{
  double G[2] = { 0.0, 0.0 }, W[4] = { 0.0, 0.0, 0.0, 0.0 }, B[4] = { 0.0, 0.0, 0.0, 0.0 }, C[4] = { 0.0, 0.0, 0.0, 0.0 };
  int s;
  if (abs(J0) != 1) info = -1;
  else if (abs(J1) != 1) info = -2;
  else info = 0;
  if (info) return;
  zscalea(A, s);
  if (s <= -3) { info = s; return; }
  U[M11] = zc(1.0, 0.0); U[M21] = zc(0.0, 0.0); U[M12] = zc(0.0, 0.0); U[M22] = zc(1.0, 0.0);
  Z[M11] = zc(1.0, 0.0); Z[M21] = zc(0.0, 0.0); Z[M12] = zc(0.0, 0.0); Z[M22] = zc(1.0, 0.0);
  zhsvd2t(A, J0, J1, U, Z, info);
  if (info > 0) {
    W[M11] = A[M11].x; W[M21] = A[M21].x; W[M12] = A[M12].x; W[M22] = A[M22].x;
    khsvd2(W, J0, J1, G, B, C, s, th1, info);
  }
  else if (info == 0) {
    if (s == 0) { W[M11] = A[M11].x; W[M22] = A[M22].x; }
    else { W[M11] = scale(A[M11].x, -s); W[M22] = scale(A[M22].x, -s); }
  }
  if (info < 0) return;
  bool th1fix = false;
  if (info > 0) {
    zc2a(B, U);
    za2c(Z, C);
    if (!(info & 8)) { W[M11] = G[0]; W[M22] = G[1]; }
    else {
      if (s != 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) A[k] = zc(scale(A[k].x, -s), scale(A[k].y, -s));
      zc2a(B, A);
      za2c(A, C);
      th1fix = true;
    }
  }
  if (!th1fix) { A[M11] = zc(W[M11], 0.0); A[M22] = zc(W[M22], 0.0); }
  zhsvd2s(A, J0, J1, U, Z, info);
}

// complex rotation coefficients: BA (src/Z/ztransf.F90:298-364) and AB / ABODNZF2 (:385-447, :478-636)
struct ZRot {
  double2 r1, r2, m1, m2;
  int c1, c2;
};

__device__ __forceinline__ ZRot zrot_ba(const double2 B[4], int quirk)
{
  ZRot t;
  t.c1 = (zabs(B[M11]) >= zabs(B[M12]));
  t.c2 = (zabs(B[M22]) >= zabs(B[M21]));
  t.r1 = t.c1 ? zratio(B[M12], B[M11]) : zratio(B[M11], B[M12]);
  t.r2 = t.c2 ? zratio(B[M21], B[M22]) : zratio(B[M22], B[M21]);
  // src/Z/ztransf.F90:325 uses R1 in the (c1, !c2) branch where src/D/dtransf.F90:155 uses R2
  if (quirk && t.c1 && !t.c2) t.r2 = t.r1;
  t.m1 = t.c1 ? B[M11] : B[M12];
  t.m2 = t.c2 ? B[M22] : B[M21];
  return t;
}

// BA applies ZZFMA(R, data, data) then ZZMUL(XX, B)
__device__ __forceinline__ void zrot_apply_ba(const ZRot &t, double2 &x, double2 &y)
{
  const double2 xx = t.c1 ? zzfma(t.r1, y, x) : zzfma(t.r1, x, y);
  const double2 yy = t.c2 ? zzfma(t.r2, x, y) : zzfma(t.r2, y, x);
  x = zzmul(xx, t.m1);
  y = zzmul(yy, t.m2);
}

__device__ __forceinline__ ZRot zrot_ab(const double2 B[4])
{
  ZRot t;
  t.c1 = (zabs(B[M11]) >= zabs(B[M21]));
  t.c2 = (zabs(B[M22]) >= zabs(B[M12]));
  t.r1 = t.c1 ? zratio(B[M21], B[M11]) : zratio(B[M11], B[M21]);
  t.r2 = t.c2 ? zratio(B[M12], B[M22]) : zratio(B[M22], B[M12]);
  t.m1 = t.c1 ? B[M11] : B[M21];
  t.m2 = t.c2 ? B[M22] : B[M12];
  return t;
}

// AB and ABODNZF2 apply ZZFMA(data, R, data) then ZZMUL(XX, B)
__device__ __forceinline__ void zrot_apply_ab(const ZRot &t, double2 &x, double2 &y)
{
  const double2 xx = t.c1 ? zzfma(y, t.r1, x) : zzfma(x, t.r1, y);
  const double2 yy = t.c2 ? zzfma(x, t.r2, y) : zzfma(y, t.r2, x);
  x = zzmul(xx, t.m1);
  y = zzmul(yy, t.m2);
}

}  // namespace jk
