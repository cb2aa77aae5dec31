// jk_math.cuh -- device scalar arithmetic of the J-Kogbetliantz step.
//
// Every routine restates the reference's Fortran operation for operation:
// FMAD(a,b,c) of the reference is a fused fma(); division and sqrt are the IEEE
// round-to-nearest operations (the library is built with -fmad=false so nothing
// else is fused); HYPOT and complex ABS are the project's own jk_hypot(); EXPONENT
// and SCALE are exact integer restatements.  Reference citations are path:line
// inside the reference project.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define JK_TH1FIX 0.75
#define JK_EH 1024
#define JK_ET (-1021)
#define JK_MINF 4.9406564584124654e-324
#define JK_HUGE 1.7976931348623157e308

// column-major 2x2 slots: (1,1) (2,1) (1,2) (2,2)
#define M11 0
#define M21 1
#define M12 2
#define M22 3

namespace jk {

__device__ __forceinline__ double twof() { return sqrt(JK_HUGE); }  // src/shared/params.F90:31

__device__ __forceinline__ bool neg(double x) { return (__double_as_longlong(x) < 0); }  // SIGN(1,x) .EQ. -1

__device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }

// Fortran EXPONENT(x): x = f*2^e with 0.5 <= |f| < 1; 0 for x = 0
__device__ __forceinline__ int exponent(double x)
{
  const unsigned long long a = (unsigned long long)__double_as_longlong(x) & 0x7FFFFFFFFFFFFFFFULL;
  if (!a) return 0;
  const int e = (int)(a >> 52);
  if (e == 0x7FF) return 0x7FFFFFFF;
  if (!e) return (64 - __clzll((long long)a)) - 1074;
  return e - 1022;
}

// Fortran SCALE(x,e) = x*2^e, correctly rounded
__device__ __forceinline__ double scale(double x, int e)
{
  const unsigned long long u = (unsigned long long)__double_as_longlong(x);
  const unsigned long long s = u & 0x8000000000000000ULL;
  const unsigned long long a = u & 0x7FFFFFFFFFFFFFFFULL;
  if (!a || ((a >> 52) == 0x7FF) || !e) return x;
  int ex = (int)(a >> 52);
  unsigned long long m = a & 0x000FFFFFFFFFFFFFULL;
  if (!ex) {
    const int sh = __clzll((long long)m) - 11;
    m <<= sh;
    ex = 1 - sh;
  }
  else
    m |= 0x0010000000000000ULL;
  const long long ne = (long long)ex + (long long)e;
  if (ne >= 0x7FF) return __longlong_as_double((long long)(s | 0x7FF0000000000000ULL));
  if (ne >= 1) return __longlong_as_double((long long)(s | ((unsigned long long)ne << 52) | (m & 0x000FFFFFFFFFFFFFULL)));
  const long long sh = 1 - ne;
  if (sh > 54) return __longlong_as_double((long long)s);
  unsigned long long q = m >> sh;
  const unsigned long long r = m & ((1ULL << sh) - 1ULL), h = 1ULL << (sh - 1);
  if ((r > h) || ((r == h) && (q & 1ULL))) ++q;
  return __longlong_as_double((long long)(s | q));
}

// project-own HYPOT: exact power-of-two scaling, h = sqrt(fma(a,a,b*b)), one Newton
// step with the residual a^2 + b^2 - h^2 assembled from error-free products
__device__ __forceinline__ double hypot2(double x, double y)
{
  const double ax = fabs(x), ay = fabs(y);
  if (isinf(ax) || isinf(ay)) return __longlong_as_double(0x7FF0000000000000LL);
  if (isnan(ax) || isnan(ay)) return ax + ay;
  const double a = (ax >= ay) ? ax : ay;
  const double b = (ax >= ay) ? ay : ax;
  if (b == 0.0) return a;
  const int ea = exponent(a);
  if ((ea - exponent(b)) > 54) return a;
  const double as = scale(a, -ea), bs = scale(b, -ea);
  double h = sqrt(fma(as, as, __dmul_rn(bs, bs)));
  const double hh = __dmul_rn(h, h), he = fma(h, h, -hh);
  const double aa = __dmul_rn(as, as), ae = fma(as, as, -aa);
  const double bb = __dmul_rn(bs, bs), be = fma(bs, bs, -bb);
  const double r = __dadd_rn(__dadd_rn(__dsub_rn(aa, hh), bb), __dsub_rn(__dadd_rn(ae, be), he));
  h = __dadd_rn(h, __ddiv_rn(r, __dadd_rn(h, h)));
  return scale(h, ea);
}

// hypot2 with the power-of-two scalings done by multiplication where that is exact: for
// finite x, y whose larger magnitude a is normal with exponent in [-999, 999] and whose
// smaller one b is normal, a * 2^-ea, b * 2^-ea and h * 2^ea are normal numbers (or, for
// the last, h * 2^ea is rounded once, as SCALE rounds), so every value equals hypot2's bit
// for bit; everything else goes through hypot2.  The same operations in the same order.
__device__ __forceinline__ double hypot2_fast(double x, double y)
{
  const double ax = fabs(x), ay = fabs(y);
  const double a = (ax >= ay) ? ax : ay;
  const double b = (ax >= ay) ? ay : ax;
  const int ba = (int)((unsigned long long)__double_as_longlong(a) >> 52);
  const int bb = (int)((unsigned long long)__double_as_longlong(b) >> 52);
  if (ba >= 23 && ba <= 2021 && bb >= 1 && ax == ax && ay == ay) {
    const int ea = ba - 1022;
    if (ea - (bb - 1022) > 54) return a;
    const double f = __longlong_as_double((long long)(1023 - ea) << 52);
    const double g = __longlong_as_double((long long)(1023 + ea) << 52);
    const double as = __dmul_rn(a, f), bs = __dmul_rn(b, f);
    double h = sqrt(fma(as, as, __dmul_rn(bs, bs)));
    const double hh = __dmul_rn(h, h), he = fma(h, h, -hh);
    const double aa = __dmul_rn(as, as), ae = fma(as, as, -aa);
    const double bq = __dmul_rn(bs, bs), be = fma(bs, bs, -bq);
    const double r = __dadd_rn(__dadd_rn(__dsub_rn(aa, hh), bq), __dsub_rn(__dadd_rn(ae, be), he));
    h = __dadd_rn(h, __ddiv_rn(r, __dadd_rn(h, h)));
    return __dmul_rn(h, g);
  }
  return hypot2(x, y);
}

// QUIET_NAN, src/shared/utils.F90:144-149
__device__ __forceinline__ double quiet_nan(long long payload)
{
  return __longlong_as_double((long long)((unsigned long long)payload | 0x7FF8000000000000ULL));
}

// DASUM2, src/D/dtransf.F90:12-38
__device__ __forceinline__ double dasum2(double x1, double x2)
{
  const double a = fabs(x1), b = fabs(x2);
  if (a >= b) {
    if (a == 0.0) return 0.0;
    return __dmul_rn(fma(b, __ddiv_rn(b, a), a), a);
  }
  return __dmul_rn(fma(a, __ddiv_rn(a, b), b), b);
}

// DASUM4, src/Z/ztransf.F90:18-75
__device__ __forceinline__ double dasum4(double x1, double x2, double x3, double x4)
{
  double x0 = fabs(x1), xa = fabs(x2), xb = fabs(x3), xc = fabs(x4);
  double y0, y1, y2, y3;
  if (x0 <= xa) { y0 = x0; y1 = xa; } else { y0 = xa; y1 = x0; }
  if (xb <= xc) { y2 = xb; y3 = xc; } else { y2 = xc; y3 = xb; }
  double z0, z1, z2, z3;
  if (y0 <= y2) { z0 = y0; z1 = y2; } else { z0 = y2; z1 = y0; }
  if (y1 <= y3) { z2 = y1; z3 = y3; } else { z2 = y3; z3 = y1; }
  double w1, w2;
  if (z1 <= z2) { w1 = z1; w2 = z2; } else { w1 = z2; w2 = z1; }
  double s = __dmul_rn(z0, z0);
  s = fma(w1, w1, s);
  s = fma(w2, w2, s);
  s = fma(z3, z3, s);
  return s;
}

// ------------------------------------------------------------------------
// shared triangular 2x2 kernels, src/shared/ktransf.F90
// ------------------------------------------------------------------------

// KHSVD2T, src/shared/ktransf.F90:15-55
__device__ __forceinline__ void khsvd2t(const double A[4], double G[2], double U[4], double Z[4], int s)
{
  double x = fmax(__ddiv_rn(A[M12], A[M11]), 0.0);
  double y = fmax(__ddiv_rn(A[M22], A[M11]), 0.0);
  const double t2 = fmin(fmax(__ddiv_rn(__dmul_rn(scale(fmin(x, y), 1), fmax(x, y)), fma(__dsub_rn(x, y), __dadd_rn(x, y), 1.0)), 0.0), twof());
  const double tu = __ddiv_rn(t2, __dadd_rn(1.0, sqrt(fma(t2, t2, 1.0))));
  const double cu = sqrt(fma(tu, tu, 1.0));
  const double tz = fma(y, tu, x);
  const double cz = sqrt(fma(tz, tz, 1.0));
  int d, e;
  y = __ddiv_rn(cz, cu);
  x = y;
  d = exponent(x) - JK_ET;
  if (s > d) { x = scale(x, -d); e = s - d; }
  else { x = scale(x, -s); e = 0; }
  G[0] = __dmul_rn(scale(A[M11], -e), x);
  G[1] = scale(__ddiv_rn(A[M22], y), -s);
  U[M11] = cu; U[M21] = -tu; U[M12] = tu; U[M22] = cu;
  Z[M11] = cz; Z[M21] = tz; Z[M12] = -tz; Z[M22] = cz;
}

// KHSVD2U, src/shared/ktransf.F90:59-112
__device__ __forceinline__ void khsvd2u(const double A[4], double G[2], double U[4], double Z[4], int s, double th1, int &info)
{
  double x = fmax(__ddiv_rn(A[M12], A[M11]), 0.0);
  double y = fmax(__ddiv_rn(A[M22], A[M11]), 0.0);
  double t2 = -fmin(fmax(__ddiv_rn(__dmul_rn(scale(fmin(x, y), 1), fmax(x, y)), fma(__dsub_rn(y, x), __dadd_rn(y, x), 1.0)), 0.0), twof());
  const double tu = __ddiv_rn(t2, __dadd_rn(1.0, sqrt(fma(t2, t2, 1.0))));
  double tz = -fma(y, tu, x);
  int d, e;
  t2 = fabs(tz);
  if (t2 >= 1.0) { info = -10; return; }
  if (t2 >= th1) { tz = copysign(JK_TH1FIX, tz); info += 8; }
  const double cu = sqrt(fma(tu, tu, 1.0));
  const double cz = sqrt(fma(-tz, tz, 1.0));
  if (t2 < th1) {
    y = __ddiv_rn(cu, cz);
    x = y;
    d = exponent(x) - JK_ET;
    if (s > d) { x = scale(x, -d); e = s - d; }
    else { x = scale(x, -s); e = 0; }
    G[0] = scale(__ddiv_rn(A[M11], y), -s);
    G[1] = __dmul_rn(scale(A[M22], -e), x);
  }
  U[M11] = cu; U[M21] = -tu; U[M12] = tu; U[M22] = cu;
  Z[M11] = cz; Z[M21] = tz; Z[M12] = tz; Z[M22] = cz;
}

// KHSVD2L, src/shared/ktransf.F90:116-169
__device__ __forceinline__ void khsvd2l(const double A[4], double G[2], double U[4], double Z[4], int s, double th1, int &info)
{
  double x = fmax(__ddiv_rn(A[M21], A[M22]), 0.0);
  double y = fmax(__ddiv_rn(A[M11], A[M22]), 0.0);
  double t2 = fmin(fmax(__ddiv_rn(__dmul_rn(scale(fmin(x, y), 1), fmax(x, y)), fma(__dsub_rn(y, x), __dadd_rn(y, x), 1.0)), 0.0), twof());
  const double tu = __ddiv_rn(t2, __dadd_rn(1.0, sqrt(fma(t2, t2, 1.0))));
  double tz = fma(y, tu, -x);
  int d, e;
  t2 = fabs(tz);
  if (t2 >= 1.0) { info = -11; return; }
  if (t2 >= th1) { tz = copysign(JK_TH1FIX, tz); info += 8; }
  const double cu = sqrt(fma(tu, tu, 1.0));
  const double cz = sqrt(fma(-tz, tz, 1.0));
  if (t2 < th1) {
    y = __ddiv_rn(cu, cz);
    x = y;
    d = exponent(x) - JK_ET;
    if (s > d) { x = scale(x, -d); e = s - d; }
    else { x = scale(x, -s); e = 0; }
    G[0] = __dmul_rn(scale(A[M11], -e), x);
    G[1] = scale(__ddiv_rn(A[M22], y), -s);
  }
  U[M11] = cu; U[M21] = -tu; U[M12] = tu; U[M22] = cu;
  Z[M11] = cz; Z[M21] = tz; Z[M12] = tz; Z[M22] = cz;
}

// KHSVD2 (argument-checking form), src/shared/ktransf.F90:173-217
__device__ __forceinline__ void khsvd2(const double A[4], const int J0, const int J1, double G[2], double U[4], double Z[4], int s, double th1, int &info)
{
  if ((info != 0) && (info != 1)) info = -1;
  else if (abs(J0) != 1) info = -2;
  else if (abs(J1) != 1) info = -3;
  else if (!(A[M11] >= 0.0)) info = -4;
  else if (!(A[M21] >= 0.0)) info = -5;
  else if (!(A[M12] >= 0.0)) info = -6;
  else if (!(A[M22] >= 0.0)) info = -7;
  else if (A[M21] == 0.0) {
    if (J0 == J1) { if (info == 1) khsvd2t(A, G, U, Z, s); }
    else { if (info == 1) khsvd2u(A, G, U, Z, s, th1, info); }
  }
  else if (A[M12] == 0.0) {
    if (J0 == J1) info = -8;
    else if (info == 1) khsvd2l(A, G, U, Z, s, th1, info);
  }
  else info = -9;
}

// ------------------------------------------------------------------------
// real 2x2 HSVD, src/D/dtransf.F90
// ------------------------------------------------------------------------

__device__ __forceinline__ void dswap(double &a, double &b) { const double t = a; a = b; b = t; }

// C1A, src/D/dtransf.F90:73-83
__device__ __forceinline__ void c1a(const double B[4], double &a1, double &a2)
{
  const double c1 = __ddiv_rn(fma(B[M12], a2, a1), B[M11]);
  const double c2 = __ddiv_rn(fma(B[M21], a1, a2), B[M22]);
  a1 = c1; a2 = c2;
}

// C2A, src/D/dtransf.F90:87-100
__device__ __forceinline__ void c2a(const double B[4], double A[4])
{
  double C[4];
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    C[2 * j + 0] = __ddiv_rn(fma(B[M12], A[2 * j + 1], A[2 * j + 0]), B[M11]);
    C[2 * j + 1] = __ddiv_rn(fma(B[M21], A[2 * j + 0], A[2 * j + 1]), B[M22]);
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) A[k] = C[k];
}

// A2C, src/D/dtransf.F90:104-117
__device__ __forceinline__ void a2c(double A[4], const double B[4])
{
  double C[4];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    C[i + 0] = __ddiv_rn(fma(A[i + 2], B[M21], A[i + 0]), B[M11]);
    C[i + 2] = __ddiv_rn(fma(A[i + 0], B[M12], A[i + 2]), B[M22]);
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) A[k] = C[k];
}

// DHSVD2T, src/D/dtransf.F90:352-532
__device__ __forceinline__ void dhsvd2t(double A[4], const int J0, const int J1, double U[4], double Z[4], int &info)
{
  double c, s, r;
  bool p, d = true;
  if (A[M21] == 0.0) c = fabs(A[M11]);
  else if (A[M11] == 0.0) { c = fabs(A[M21]); d = false; }
  else { c = hypot2(A[M11], A[M21]); d = false; }
  if (A[M12] == 0.0) s = fabs(A[M22]);
  else if (A[M22] == 0.0) { s = fabs(A[M12]); d = false; }
  else { s = hypot2(A[M12], A[M22]); d = false; }

  if (c < s) {
    r = s;
    dswap(A[M11], A[M12]); dswap(A[M21], A[M22]);
    if (J0 == J1) { dswap(Z[M11], Z[M12]); dswap(Z[M21], Z[M22]); }
    p = true;
  }
  else { r = c; p = false; }

  if (neg(A[M11])) { U[M11] = -U[M11]; U[M12] = -U[M12]; A[M12] = -A[M12]; A[M11] = -A[M11]; }
  if (neg(A[M21])) { U[M21] = -U[M21]; U[M22] = -U[M22]; A[M22] = -A[M22]; A[M21] = -A[M21]; }

  if (A[M11] < A[M21]) {
    dswap(U[M11], U[M21]); dswap(U[M12], U[M22]);
    dswap(A[M11], A[M21]); dswap(A[M12], A[M22]);
  }

  if (!d) {
    s = __ddiv_rn(A[M21], A[M11]);
    c = sqrt(fma(s, s, 1.0));
    const double Q[4] = { c, -s, s, c };
    c2a(Q, U);
    c1a(Q, A[M12], A[M22]);
  }
  A[M11] = r;
  A[M21] = 0.0;

  if ((J0 != J1) && p) {
    dswap(A[M11], A[M12]); dswap(A[M21], A[M22]);
    dswap(U[M11], U[M21]); dswap(U[M12], U[M22]);
    dswap(A[M11], A[M21]); dswap(A[M12], A[M22]);
    if (neg(A[M21])) { Z[M11] = -Z[M11]; Z[M21] = -Z[M21]; A[M11] = -A[M11]; A[M21] = -A[M21]; }
    if (neg(A[M11])) { U[M11] = -U[M11]; U[M12] = -U[M12]; A[M11] = -A[M11]; }
  }
  else {
    if (neg(A[M12])) { Z[M12] = -Z[M12]; Z[M22] = -Z[M22]; A[M22] = -A[M22]; A[M12] = -A[M12]; }
    if (neg(A[M22])) { U[M21] = -U[M21]; U[M22] = -U[M22]; A[M22] = -A[M22]; }
  }
  info = d ? 0 : 1;
}

// DHSVD2S, src/D/dtransf.F90:536-577 (A(2,1), A(1,2) are the temporaries, as there)
__device__ __forceinline__ void dhsvd2s(double A[4], const int J0, const int J1, double U[4], double Z[4], int &info)
{
  const int t = J0 + J1;
  if (((t == 2) && (A[M11] < A[M22])) || ((t == -2) && (A[M22] < A[M11]))) {
    A[M21] = U[M11]; A[M12] = U[M12];
    U[M11] = U[M21]; U[M12] = U[M22];
    U[M21] = A[M21]; U[M22] = A[M12];
    A[M21] = A[M11]; A[M11] = A[M22]; A[M22] = A[M21];
    A[M21] = Z[M11]; A[M12] = Z[M21];
    Z[M11] = Z[M12]; Z[M21] = Z[M22];
    Z[M12] = A[M21]; Z[M22] = A[M12];
  }
  if (!(info & 8)) { A[M21] = 0.0; A[M12] = 0.0; }
  if ((U[M11] != 1.0) || (U[M21] != 0.0) || (U[M12] != 0.0) || (U[M22] != 1.0)) info += 2;
  if ((Z[M11] != 1.0) || (Z[M21] != 0.0) || (Z[M12] != 0.0) || (Z[M22] != 1.0)) info += 4;
}

// DSCALEA, src/D/dtransf.F90:581-610
__device__ __forceinline__ void dscalea(double A[4], int &s)
{
  s = 0x7FFFFFFF;
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const double aa = fabs(A[2 * j + i]);
      if (!(aa <= JK_HUGE)) { s = -((j + 1) * 2 + (i + 1)); return; }
      s = imin(s, JK_EH - exponent(fmax(aa, JK_MINF)) - 2);
    }
  if (s != 0)
#pragma unroll
    for (int k = 0; k < 4; ++k) A[k] = scale(A[k], s);
}

// DHSVD2 (argument-checking form), src/D/dtransf.F90:614-683
__device__ __forceinline__ void dhsvd2(double A[4], const int J0, const int J1, double U[4], double Z[4], double th1, int &info)
{
  double G[2] = { 0.0, 0.0 }, B[4] = { 0.0, 0.0, 0.0, 0.0 }, C[4] = { 0.0, 0.0, 0.0, 0.0 };
  int s;
  if (abs(J0) != 1) info = -1;
  else if (abs(J1) != 1) info = -2;
  else info = 0;
  if (info) return;
  dscalea(A, s);
  if (s <= -3) { info = s; return; }
  U[M11] = 1.0; U[M21] = 0.0; U[M12] = 0.0; U[M22] = 1.0;
  Z[M11] = 1.0; Z[M21] = 0.0; Z[M12] = 0.0; Z[M22] = 1.0;
  dhsvd2t(A, J0, J1, U, Z, info);
  if (info > 0) khsvd2(A, J0, J1, G, B, C, s, th1, info);
  else if ((info == 0) && (s != 0)) { A[M11] = scale(A[M11], -s); A[M22] = scale(A[M22], -s); }
  if (info < 0) return;
  if (info > 0) {
    c2a(B, U);
    a2c(Z, C);
    if (!(info & 8)) { A[M11] = G[0]; A[M22] = G[1]; }
    else {
#pragma unroll
      for (int k = 0; k < 4; ++k) A[k] = scale(A[k], -s);
      c2a(B, A);
      a2c(A, C);
    }
  }
  dhsvd2s(A, J0, J1, U, Z, info);
}

// ------------------------------------------------------------------------
// the branch-selected scaled rotation of BA / AB / ABODNDF2
// (src/D/dtransf.F90:121-348):  with flags c1, c2, ratios r1, r2, multipliers m1, m2,
//   xx = c1 ? fma(r1, y, x) : fma(r1, x, y);   x' = xx * m1
//   yy = c2 ? fma(r2, x, y) : fma(r2, y, x);   y' = yy * m2
// ------------------------------------------------------------------------
struct Rot {
  double r1, r2, m1, m2;
  int c1, c2;
};

// coefficients of BA(B, ...) (rows), src/D/dtransf.F90:140-182
__device__ __forceinline__ Rot rot_ba(const double B[4])
{
  Rot t;
  t.c1 = (fabs(B[M11]) >= fabs(B[M12]));
  t.c2 = (fabs(B[M22]) >= fabs(B[M21]));
  t.r1 = t.c1 ? __ddiv_rn(B[M12], B[M11]) : __ddiv_rn(B[M11], B[M12]);
  t.r2 = t.c2 ? __ddiv_rn(B[M21], B[M22]) : __ddiv_rn(B[M22], B[M21]);
  t.m1 = t.c1 ? B[M11] : B[M12];
  t.m2 = t.c2 ? B[M22] : B[M21];
  return t;
}

// coefficients of AB(B, ...) (columns) and ABODNDF2, src/D/dtransf.F90:203-241, 261-347
__device__ __forceinline__ Rot rot_ab(const double B[4])
{
  Rot t;
  t.c1 = (fabs(B[M11]) >= fabs(B[M21]));
  t.c2 = (fabs(B[M22]) >= fabs(B[M12]));
  t.r1 = t.c1 ? __ddiv_rn(B[M21], B[M11]) : __ddiv_rn(B[M11], B[M21]);
  t.r2 = t.c2 ? __ddiv_rn(B[M12], B[M22]) : __ddiv_rn(B[M22], B[M12]);
  t.m1 = t.c1 ? B[M11] : B[M21];
  t.m2 = t.c2 ? B[M22] : B[M12];
  return t;
}

__device__ __forceinline__ void rot_apply(const Rot &t, double &x, double &y)
{
  const double xx = t.c1 ? fma(t.r1, y, x) : fma(t.r1, x, y);
  const double yy = t.c2 ? fma(t.r2, x, y) : fma(t.r2, y, x);
  x = __dmul_rn(xx, t.m1);
  y = __dmul_rn(yy, t.m2);
}

// ------------------------------------------------------------------------
// complex helpers, src/Z/ztransf.F90:79-227 (a complex number is a double2 (re, im))
// ------------------------------------------------------------------------
__device__ __forceinline__ double2 zc(double re, double im) { return make_double2(re, im); }
__device__ __forceinline__ double2 conj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 zneg(double2 a) { return make_double2(-a.x, -a.y); }
__device__ __forceinline__ bool zeq0(double2 a) { return (a.x == 0.0) && (a.y == 0.0); }
__device__ __forceinline__ bool zne1(double2 a) { return (a.x != 1.0) || (a.y != 0.0); }
__device__ __forceinline__ double zabs(double2 a) { return hypot2(a.x, a.y); }
__device__ __forceinline__ double zabs_fast(double2 a) { return hypot2_fast(a.x, a.y); }

// ZDFMA, src/Z/ztransf.F90:130-141
__device__ __forceinline__ double2 zdfma(double a, double2 b, double2 c) { return zc(fma(a, b.x, c.x), fma(a, b.y, c.y)); }

// ZZFMA, src/Z/ztransf.F90:162-174 (argument order matters)
__device__ __forceinline__ double2 zzfma(double2 a, double2 b, double2 c)
{
  double f = fma(-a.y, b.y, c.x);
  const double r = fma(a.x, b.x, f);
  f = fma(a.y, b.x, c.y);
  return zc(r, fma(a.x, b.y, f));
}

// ZZMUL, src/Z/ztransf.F90:193-205 (argument order matters)
__device__ __forceinline__ double2 zzmul(double2 a, double2 b)
{
  double f = __dmul_rn(a.y, b.y);
  const double r = fma(a.x, b.x, -f);
  f = __dmul_rn(a.y, b.x);
  return zc(r, fma(a.x, b.y, f));
}

// ZDDIV, src/Z/ztransf.F90:209-215
__device__ __forceinline__ double2 zddiv(double2 a, double b) { return zc(__ddiv_rn(a.x, b), __ddiv_rn(a.y, b)); }

// ZZDIV, src/Z/ztransf.F90:220-227
__device__ __forceinline__ double2 zzdiv(double2 a, double2 b)
{
  const double f = zabs(b);
  return zddiv(zzmul(conj(zddiv(b, f)), a), f);
}

__device__ __forceinline__ double2 zratio(double2 num, double2 den)
{
  return (den.y == 0.0) ? zddiv(num, den.x) : zzdiv(num, den);
}

}  // namespace jk
