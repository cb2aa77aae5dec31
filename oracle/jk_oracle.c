/*
 * jk_oracle.c -- TEST INFRASTRUCTURE ONLY: CPU restatement of venovako/JKogb's
 * real step loop (djk) and of the parts shared with the complex loop.
 * Only tests/, the smoke check and the benchmark's CPU-baseline leg use it.
 *
 * Every function cites the reference routine (path:line within the reference
 * project) whose arithmetic it restates, operation for operation.
 */
#include "jk_oracle_impl.h"

/* ------------------------------------------------------------------------- */
/* scalar helpers                                                            */
/* ------------------------------------------------------------------------- */

static inline uint64_t jo_bits(double x) { uint64_t u; memcpy(&u, &x, 8); return u; }
static inline double jo_from_bits(uint64_t u) { double x; memcpy(&x, &u, 8); return x; }

/* QUIET_NAN, src/shared/utils.F90:144-149 */
double jo_quiet_nan(int64_t payload)
{
  return jo_from_bits((uint64_t)payload | UINT64_C(0x7FF8000000000000));
}

/* Fortran EXPONENT(x): the e with x = f*2^e, 0.5 <= |f| < 1; 0 for x = 0. */
int jo_exponent(double x)
{
  const uint64_t a = jo_bits(x) & UINT64_C(0x7FFFFFFFFFFFFFFF);
  if (!a)
    return 0;
  const int e = (int)(a >> 52);
  if (e == 0x7FF)
    return INT_MAX;
  if (!e)
    return (64 - __builtin_clzll(a)) - 1074;
  return e - 1022;
}

/* Fortran SCALE(x,e) = x*2^e, correctly rounded (one rounding into the subnormals). */
double jo_scale(double x, int e)
{
  const uint64_t u = jo_bits(x);
  const uint64_t s = u & UINT64_C(0x8000000000000000);
  const uint64_t a = u & UINT64_C(0x7FFFFFFFFFFFFFFF);
  if (!a || ((a >> 52) == 0x7FF) || !e)
    return x;
  int ex = (int)(a >> 52);
  uint64_t m = a & UINT64_C(0x000FFFFFFFFFFFFF);
  if (!ex) {
    const int sh = __builtin_clzll(m) - 11;
    m <<= sh;
    ex = 1 - sh;
  }
  else
    m |= UINT64_C(0x0010000000000000);
  const long ne = (long)ex + (long)e;
  if (ne >= 0x7FF)
    return jo_from_bits(s | UINT64_C(0x7FF0000000000000));
  if (ne >= 1)
    return jo_from_bits(s | ((uint64_t)ne << 52) | (m & UINT64_C(0x000FFFFFFFFFFFFF)));
  const long sh = 1 - ne;
  if (sh > 54)
    return jo_from_bits(s);
  uint64_t q = m >> sh;
  const uint64_t r = m & ((UINT64_C(1) << sh) - 1u), h = UINT64_C(1) << (sh - 1);
  if ((r > h) || ((r == h) && (q & 1u)))
    ++q;
  return jo_from_bits(s | q);
}

/*
 * Project-own HYPOT (the reference calls the Fortran intrinsic, i.e. libm).
 * max/min ordering, exact power-of-two scaling, h = sqrt(fma(a,a,b*b)), then one
 * Newton step h += r/(2h) with the residual r = a^2 + b^2 - h^2 assembled from
 * error-free products.  The same operation sequence runs on the GPU.
 */
double jo_hypot(double x, double y)
{
  const double ax = fabs(x), ay = fabs(y);
  if (isinf(ax) || isinf(ay))
    return INFINITY;
  if (isnan(ax) || isnan(ay))
    return ax + ay;
  const double a = (ax >= ay) ? ax : ay;
  const double b = (ax >= ay) ? ay : ax;
  if (b == 0.0)
    return a;
  const int ea = jo_exponent(a);
  if ((ea - jo_exponent(b)) > 54)
    return a;
  const double as = jo_scale(a, -ea), bs = jo_scale(b, -ea);
  double h = sqrt(fma(as, as, bs * bs));
  const double hh = h * h, he = fma(h, h, -hh);
  const double aa = as * as, ae = fma(as, as, -aa);
  const double bb = bs * bs, be = fma(bs, bs, -bb);
  const double r = ((aa - hh) + bb) + ((ae + be) - he);
  h = h + r / (h + h);
  return jo_scale(h, ea);
}

/* DASUM2, src/D/dtransf.F90:12-38 (the non-USE_TEST branch) */
double jo_dasum2(double x1, double x2)
{
  const double a = fabs(x1), b = fabs(x2);
  if (a >= b) {
    if (a == 0.0)
      return 0.0;
    return fma(b, (b / a), a) * a;
  }
  return fma(a, (a / b), b) * b;
}

/* DASUM4, src/Z/ztransf.F90:18-75 */
double jo_dasum4(double x1, double x2, double x3, double x4)
{
  double x[4] = { fabs(x1), fabs(x2), fabs(x3), fabs(x4) }, y[4];
  if (x[0] <= x[1]) { y[0] = x[0]; y[1] = x[1]; } else { y[0] = x[1]; y[1] = x[0]; }
  if (x[2] <= x[3]) { y[2] = x[2]; y[3] = x[3]; } else { y[2] = x[3]; y[3] = x[2]; }
  if (y[0] <= y[2]) { x[0] = y[0]; x[1] = y[2]; } else { x[0] = y[2]; x[1] = y[0]; }
  if (y[1] <= y[3]) { x[2] = y[1]; x[3] = y[3]; } else { x[2] = y[3]; x[3] = y[1]; }
  y[0] = x[0];
  if (x[1] <= x[2]) { y[1] = x[1]; y[2] = x[2]; } else { y[1] = x[2]; y[2] = x[1]; }
  y[3] = x[3];
  double s = y[0] * y[0];
  s = fma(y[1], y[1], s);
  s = fma(y[2], y[2], s);
  s = fma(y[3], y[3], s);
  return s;
}

/* ------------------------------------------------------------------------- */
/* shared triangular 2x2 kernels, src/shared/ktransf.F90                      */
/* ------------------------------------------------------------------------- */

/* KHSVD2T, src/shared/ktransf.F90:15-55 */
static void jo_khsvd2t(const double A[4], double G[2], double U[4], double Z[4], int s)
{
  double x = fmax(A[M12] / A[M11], 0.0);
  double y = fmax(A[M22] / A[M11], 0.0);
  const double t2 = fmin(fmax((jo_scale(fmin(x, y), 1) * fmax(x, y)) / fma((x - y), (x + y), 1.0), 0.0), jo_twof());
  const double tu = t2 / (1.0 + sqrt(fma(t2, t2, 1.0)));
  const double cu = sqrt(fma(tu, tu, 1.0));
  const double tz = fma(y, tu, x);
  const double cz = sqrt(fma(tz, tz, 1.0));
  int d, e;

  y = cz / cu;
  x = y;
  d = jo_exponent(x) - JO_ET;
  if (s > d) { x = jo_scale(x, -d); e = s - d; }
  else { x = jo_scale(x, -s); e = 0; }

  G[0] = jo_scale(A[M11], -e) * x;
  G[1] = jo_scale(A[M22] / y, -s);

  U[M11] = cu; U[M21] = -tu; U[M12] = tu; U[M22] = cu;
  Z[M11] = cz; Z[M21] = tz; Z[M12] = -tz; Z[M22] = cz;
}

/* KHSVD2U, src/shared/ktransf.F90:59-112 */
static void jo_khsvd2u(const double A[4], double G[2], double U[4], double Z[4], int s, double th1, int *info)
{
  double x = fmax(A[M12] / A[M11], 0.0);
  double y = fmax(A[M22] / A[M11], 0.0);
  double t2 = -fmin(fmax((jo_scale(fmin(x, y), 1) * fmax(x, y)) / fma((y - x), (y + x), 1.0), 0.0), jo_twof());
  const double tu = t2 / (1.0 + sqrt(fma(t2, t2, 1.0)));
  double tz = -fma(y, tu, x);
  int d, e;

  t2 = fabs(tz);
  if (t2 >= 1.0) { *info = -10; return; }
  if (t2 >= th1) { tz = copysign(JO_TH1FIX, tz); *info += 8; }
  const double cu = sqrt(fma(tu, tu, 1.0));
  const double cz = sqrt(fma(-tz, tz, 1.0));

  if (t2 < th1) {
    y = cu / cz;
    x = y;
    d = jo_exponent(x) - JO_ET;
    if (s > d) { x = jo_scale(x, -d); e = s - d; }
    else { x = jo_scale(x, -s); e = 0; }
    G[0] = jo_scale(A[M11] / y, -s);
    G[1] = jo_scale(A[M22], -e) * x;
  }

  U[M11] = cu; U[M21] = -tu; U[M12] = tu; U[M22] = cu;
  Z[M11] = cz; Z[M21] = tz; Z[M12] = tz; Z[M22] = cz;
}

/* KHSVD2L, src/shared/ktransf.F90:116-169 */
static void jo_khsvd2l(const double A[4], double G[2], double U[4], double Z[4], int s, double th1, int *info)
{
  double x = fmax(A[M21] / A[M22], 0.0);
  double y = fmax(A[M11] / A[M22], 0.0);
  double t2 = fmin(fmax((jo_scale(fmin(x, y), 1) * fmax(x, y)) / fma((y - x), (y + x), 1.0), 0.0), jo_twof());
  const double tu = t2 / (1.0 + sqrt(fma(t2, t2, 1.0)));
  double tz = fma(y, tu, -x);
  int d, e;

  t2 = fabs(tz);
  if (t2 >= 1.0) { *info = -11; return; }
  if (t2 >= th1) { tz = copysign(JO_TH1FIX, tz); *info += 8; }
  const double cu = sqrt(fma(tu, tu, 1.0));
  const double cz = sqrt(fma(-tz, tz, 1.0));

  if (t2 < th1) {
    y = cu / cz;
    x = y;
    d = jo_exponent(x) - JO_ET;
    if (s > d) { x = jo_scale(x, -d); e = s - d; }
    else { x = jo_scale(x, -s); e = 0; }
    G[0] = jo_scale(A[M11], -e) * x;
    G[1] = jo_scale(A[M22] / y, -s);
  }

  U[M11] = cu; U[M21] = -tu; U[M12] = tu; U[M22] = cu;
  Z[M11] = cz; Z[M21] = tz; Z[M12] = tz; Z[M22] = cz;
}

/* KHSVD2 (argument-checking build), src/shared/ktransf.F90:173-217 */
static void jo_khsvd2(const double A[4], const int J[2], double G[2], double U[4], double Z[4], int s, double th1, int *info)
{
  if ((*info != 0) && (*info != 1)) *info = -1;
  else if (abs(J[0]) != 1) *info = -2;
  else if (abs(J[1]) != 1) *info = -3;
  else if (!(A[M11] >= 0.0)) *info = -4;
  else if (!(A[M21] >= 0.0)) *info = -5;
  else if (!(A[M12] >= 0.0)) *info = -6;
  else if (!(A[M22] >= 0.0)) *info = -7;
  else if (A[M21] == 0.0) {
    if (J[0] == J[1]) { if (*info == 1) jo_khsvd2t(A, G, U, Z, s); }
    else { if (*info == 1) jo_khsvd2u(A, G, U, Z, s, th1, info); }
  }
  else if (A[M12] == 0.0) {
    if (J[0] == J[1]) *info = -8;
    else if (*info == 1) jo_khsvd2l(A, G, U, Z, s, th1, info);
  }
  else *info = -9;
}

/* ------------------------------------------------------------------------- */
/* real 2x2 HSVD, src/D/dtransf.F90                                          */
/* ------------------------------------------------------------------------- */

/* C1A, src/D/dtransf.F90:73-83 (A is the column (a1,a2)) */
static void jo_c1a(const double B[4], double *a1, double *a2)
{
  const double c1 = fma(B[M12], *a2, *a1) / B[M11];
  const double c2 = fma(B[M21], *a1, *a2) / B[M22];
  *a1 = c1; *a2 = c2;
}

/* C2A, src/D/dtransf.F90:87-100 */
static void jo_c2a(const double B[4], double A[4])
{
  double C[4];
  for (int j = 0; j < 2; ++j) {
    C[2 * j + 0] = fma(B[M12], A[2 * j + 1], A[2 * j + 0]) / B[M11];
    C[2 * j + 1] = fma(B[M21], A[2 * j + 0], A[2 * j + 1]) / B[M22];
  }
  memcpy(A, C, sizeof(C));
}

/* A2C, src/D/dtransf.F90:104-117 */
static void jo_a2c(double A[4], const double B[4])
{
  double C[4];
  for (int i = 0; i < 2; ++i) {
    C[i + 0] = fma(A[i + 2], B[M21], A[i + 0]) / B[M11];
    C[i + 2] = fma(A[i + 0], B[M12], A[i + 2]) / B[M22];
  }
  memcpy(A, C, sizeof(C));
}

#define JO_SWAP(a, b) do { const double t_ = (a); (a) = (b); (b) = t_; } while (0)

/* DHSVD2T, src/D/dtransf.F90:352-532 */
static void jo_dhsvd2t(double A[4], const int J[2], double U[4], double Z[4], int *info)
{
  double c, s, r, Q[4];
  bool p, d = true;

  if (A[M21] == 0.0) c = fabs(A[M11]);
  else if (A[M11] == 0.0) { c = fabs(A[M21]); d = false; }
  else { c = jo_hypot(A[M11], A[M21]); d = false; }
  if (A[M12] == 0.0) s = fabs(A[M22]);
  else if (A[M22] == 0.0) { s = fabs(A[M12]); d = false; }
  else { s = jo_hypot(A[M12], A[M22]); d = false; }

  if (c < s) {
    r = s;
    JO_SWAP(A[M11], A[M12]); JO_SWAP(A[M21], A[M22]);
    if (J[0] == J[1]) { JO_SWAP(Z[M11], Z[M12]); JO_SWAP(Z[M21], Z[M22]); }
    p = true;
  }
  else { r = c; p = false; }

  if (jo_neg(A[M11])) { U[M11] = -U[M11]; U[M12] = -U[M12]; A[M12] = -A[M12]; A[M11] = -A[M11]; }
  if (jo_neg(A[M21])) { U[M21] = -U[M21]; U[M22] = -U[M22]; A[M22] = -A[M22]; A[M21] = -A[M21]; }

  if (A[M11] < A[M21]) {
    JO_SWAP(U[M11], U[M21]); JO_SWAP(U[M12], U[M22]);
    JO_SWAP(A[M11], A[M21]); JO_SWAP(A[M12], A[M22]);
  }

  if (!d) {
    s = A[M21] / A[M11];
    c = sqrt(fma(s, s, 1.0));
    Q[M11] = c; Q[M21] = -s; Q[M12] = s; Q[M22] = c;
    jo_c2a(Q, U);
    jo_c1a(Q, &A[M12], &A[M22]);
  }
  A[M11] = r;
  A[M21] = 0.0;

  if ((J[0] != J[1]) && p) {
    JO_SWAP(A[M11], A[M12]); JO_SWAP(A[M21], A[M22]);
    JO_SWAP(U[M11], U[M21]); JO_SWAP(U[M12], U[M22]);
    JO_SWAP(A[M11], A[M21]); JO_SWAP(A[M12], A[M22]);
    if (jo_neg(A[M21])) { Z[M11] = -Z[M11]; Z[M21] = -Z[M21]; A[M11] = -A[M11]; A[M21] = -A[M21]; }
    if (jo_neg(A[M11])) { U[M11] = -U[M11]; U[M12] = -U[M12]; A[M11] = -A[M11]; }
  }
  else {
    if (jo_neg(A[M12])) { Z[M12] = -Z[M12]; Z[M22] = -Z[M22]; A[M22] = -A[M22]; A[M12] = -A[M12]; }
    if (jo_neg(A[M22])) { U[M21] = -U[M21]; U[M22] = -U[M22]; A[M22] = -A[M22]; }
  }

  *info = d ? 0 : 1;
}

/* DHSVD2S, src/D/dtransf.F90:536-577 (A(2,1), A(1,2) serve as temporaries, as there) */
static void jo_dhsvd2s(double A[4], const int J[2], double U[4], double Z[4], int *info)
{
  const int t = J[0] + J[1];
  if (((t == 2) && (A[M11] < A[M22])) || ((t == -2) && (A[M22] < A[M11]))) {
    A[M21] = U[M11]; A[M12] = U[M12];
    U[M11] = U[M21]; U[M12] = U[M22];
    U[M21] = A[M21]; U[M22] = A[M12];
    A[M21] = A[M11]; A[M11] = A[M22]; A[M22] = A[M21];
    A[M21] = Z[M11]; A[M12] = Z[M21];
    Z[M11] = Z[M12]; Z[M21] = Z[M22];
    Z[M12] = A[M21]; Z[M22] = A[M12];
  }
  if (!(*info & 8)) { A[M21] = 0.0; A[M12] = 0.0; }
  if ((U[M11] != 1.0) || (U[M21] != 0.0) || (U[M12] != 0.0) || (U[M22] != 1.0)) *info += 2;
  if ((Z[M11] != 1.0) || (Z[M21] != 0.0) || (Z[M12] != 0.0) || (Z[M22] != 1.0)) *info += 4;
}

/* DSCALEA, src/D/dtransf.F90:581-610 */
static void jo_dscalea(double A[4], int *s)
{
  *s = INT_MAX;
  for (int j = 0; j < 2; ++j)
    for (int i = 0; i < 2; ++i) {
      const double aa = fabs(A[2 * j + i]);
      if (!(aa <= DBL_MAX)) { *s = -((j + 1) * 2 + (i + 1)); return; }
      *s = jo_imin(*s, JO_EH - jo_exponent(fmax(aa, JO_MINF)) - 2);
    }
  if (*s != 0)
    for (int k = 0; k < 4; ++k)
      A[k] = jo_scale(A[k], *s);
}

/* DHSVD2 (argument-checking build), src/D/dtransf.F90:614-683 */
void jo_dhsvd2(double A[4], const int J[2], double U[4], double Z[4], double th1, int *info)
{
  double G[2] = { 0.0, 0.0 }, B[4] = { 0.0, 0.0, 0.0, 0.0 }, C[4] = { 0.0, 0.0, 0.0, 0.0 };
  int s;

  if (abs(J[0]) != 1) *info = -1;
  else if (abs(J[1]) != 1) *info = -2;
  else *info = 0;
  if (*info) return;

  jo_dscalea(A, &s);
  if (s <= -3) { *info = s; return; }

  U[M11] = 1.0; U[M21] = 0.0; U[M12] = 0.0; U[M22] = 1.0;
  Z[M11] = 1.0; Z[M21] = 0.0; Z[M12] = 0.0; Z[M22] = 1.0;

  jo_dhsvd2t(A, J, U, Z, info);
  if (*info > 0)
    jo_khsvd2(A, J, G, B, C, s, th1, info);
  else if ((*info == 0) && (s != 0)) {
    A[M11] = jo_scale(A[M11], -s);
    A[M22] = jo_scale(A[M22], -s);
  }
  if (*info < 0) return;
  if (*info > 0) {
    jo_c2a(B, U);
    jo_a2c(Z, C);
    if (!(*info & 8)) { A[M11] = G[0]; A[M22] = G[1]; }
    else {
      for (int k = 0; k < 4; ++k)
        A[k] = jo_scale(A[k], -s);
      jo_c2a(B, A);
      jo_a2c(A, C);
    }
  }
  jo_dhsvd2s(A, J, U, Z, info);
}

/* ------------------------------------------------------------------------- */
/* real rotations and the off-norm reduction                                 */
/* ------------------------------------------------------------------------- */

/* BA, src/D/dtransf.F90:121-183: rows x, y (stride lda) <- B * [x; y] */
void jo_dba(const double B[4], int n, double *x, double *y, int lda)
{
  double r1, r2, xx, yy;
  long i = 0;
  if (fabs(B[M11]) >= fabs(B[M12])) {
    r1 = B[M12] / B[M11];
    if (fabs(B[M22]) >= fabs(B[M21])) {
      r2 = B[M21] / B[M22];
      for (int j = 0; j < n; ++j, i += lda) {
        xx = fma(r1, y[i], x[i]); yy = fma(r2, x[i], y[i]);
        x[i] = xx * B[M11]; y[i] = yy * B[M22];
      }
    }
    else {
      r2 = B[M22] / B[M21];
      for (int j = 0; j < n; ++j, i += lda) {
        xx = fma(r1, y[i], x[i]); yy = fma(r2, y[i], x[i]);
        x[i] = xx * B[M11]; y[i] = yy * B[M21];
      }
    }
  }
  else {
    r1 = B[M11] / B[M12];
    if (fabs(B[M22]) >= fabs(B[M21])) {
      r2 = B[M21] / B[M22];
      for (int j = 0; j < n; ++j, i += lda) {
        xx = fma(r1, x[i], y[i]); yy = fma(r2, x[i], y[i]);
        x[i] = xx * B[M12]; y[i] = yy * B[M22];
      }
    }
    else {
      r2 = B[M22] / B[M21];
      for (int j = 0; j < n; ++j, i += lda) {
        xx = fma(r1, x[i], y[i]); yy = fma(r2, y[i], x[i]);
        x[i] = xx * B[M12]; y[i] = yy * B[M21];
      }
    }
  }
}

/* AB, src/D/dtransf.F90:187-242: columns [x y] <- [x y] * B */
void jo_dab(const double B[4], int m, double *x, double *y)
{
  double r1, r2, xx, yy;
  if (fabs(B[M11]) >= fabs(B[M21])) {
    r1 = B[M21] / B[M11];
    if (fabs(B[M22]) >= fabs(B[M12])) {
      r2 = B[M12] / B[M22];
      for (int i = 0; i < m; ++i) {
        xx = fma(y[i], r1, x[i]); yy = fma(x[i], r2, y[i]);
        x[i] = xx * B[M11]; y[i] = yy * B[M22];
      }
    }
    else {
      r2 = B[M22] / B[M12];
      for (int i = 0; i < m; ++i) {
        xx = fma(y[i], r1, x[i]); yy = fma(y[i], r2, x[i]);
        x[i] = xx * B[M11]; y[i] = yy * B[M12];
      }
    }
  }
  else {
    r1 = B[M11] / B[M21];
    if (fabs(B[M22]) >= fabs(B[M12])) {
      r2 = B[M12] / B[M22];
      for (int i = 0; i < m; ++i) {
        xx = fma(x[i], r1, y[i]); yy = fma(x[i], r2, y[i]);
        x[i] = xx * B[M21]; y[i] = yy * B[M22];
      }
    }
    else {
      r2 = B[M22] / B[M12];
      for (int i = 0; i < m; ++i) {
        xx = fma(x[i], r1, y[i]); yy = fma(y[i], r2, x[i]);
        x[i] = xx * B[M21]; y[i] = yy * B[M12];
      }
    }
  }
}

/* ABODNDF2, src/D/dtransf.F90:246-348 (p, q 1-based; rows p and q skipped) */
double jo_abodndf2(const double B[4], int m, const double *x, const double *y, double aqp, double apq, int p, int q)
{
  double r1, r2, xx, yy, d = 0.0;
  d = fma(x[q - 1] - aqp, x[q - 1] + aqp, d);
  d = fma(y[p - 1] - apq, y[p - 1] + apq, d);
  const int c1 = (fabs(B[M11]) >= fabs(B[M21]));
  const int c2 = (fabs(B[M22]) >= fabs(B[M12]));
  r1 = c1 ? (B[M21] / B[M11]) : (B[M11] / B[M21]);
  r2 = c2 ? (B[M12] / B[M22]) : (B[M22] / B[M12]);
  for (int i = 0; i < m; ++i) {
    if ((i == p - 1) || (i == q - 1))
      continue;
    if (c1) xx = fma(y[i], r1, x[i]) * B[M11];
    else xx = fma(x[i], r1, y[i]) * B[M21];
    if (c2) yy = fma(x[i], r2, y[i]) * B[M22];
    else yy = fma(y[i], r2, x[i]) * B[M12];
    d = fma((x[i] - xx), (x[i] + xx), d);
    d = fma((y[i] - yy), (y[i] + yy), d);
  }
  return d;
}

/* ------------------------------------------------------------------------- */
/* pair weights, src/D/dstep.F90:12-72                                       */
/* ------------------------------------------------------------------------- */

#define AE(A, lda, i, j) ((A)[(long)((j) - 1) * (lda) + ((i) - 1)])

/* DMAGF2T, src/D/dstep.F90:12-37 (p, q 1-based) */
double jo_dmagf2t(int n, int p, int q, const double *A, int lda, const int *J)
{
  const double app = AE(A, lda, p, p), aqp = AE(A, lda, q, p), apq = AE(A, lda, p, q), aqq = AE(A, lda, q, q);
  switch (J[p - 1] + J[q - 1]) {
  case -2:
    if ((aqp != 0.0) || (apq != 0.0) || jo_neg(app) || jo_neg(aqq) || (aqq < app))
      return jo_dasum2(aqp, apq);
    return jo_quiet_nan((int64_t)(p - 1) * n + (q - 1));
  case 2:
    if ((aqp != 0.0) || (apq != 0.0) || jo_neg(app) || jo_neg(aqq) || (app < aqq))
      return jo_dasum2(aqp, apq);
    return jo_quiet_nan((int64_t)(p - 1) * n + (q - 1));
  default:
    return jo_quiet_nan((int64_t)(p - 1) * n + (q - 1));
  }
}

/* DMAGF2H, src/D/dstep.F90:41-72 */
double jo_dmagf2h(int n, int p, int q, const double *A, int lda, const int *J)
{
  const double app = AE(A, lda, p, p), aqp = AE(A, lda, q, p), apq = AE(A, lda, p, q), aqq = AE(A, lda, q, q);
  if ((aqp != 0.0) || (apq != 0.0) || jo_neg(app) || jo_neg(aqq)) {
    double A2[4] = { app, aqp, apq, aqq }, U2[4], Z2[4];
    const int J2[2] = { J[p - 1], J[q - 1] };
    int info = 0;
    jo_dhsvd2(A2, J2, U2, Z2, JO_TH1FIX, &info);
    if (info < 0) return jo_quiet_nan((int64_t)(p - 1) * n + (q - 1));
    if (!(info & 1)) return 0.0;
    if (!(info & 4)) return jo_dasum2(aqp, apq);
    if (!(info & 8))
      return jo_abodndf2(Z2, n, &AE(A, lda, 1, p), &AE(A, lda, 1, q), 0.0, 0.0, p, q);
    return jo_abodndf2(Z2, n, &AE(A, lda, 1, p), &AE(A, lda, 1, q), A2[M21], A2[M12], p, q);
  }
  return jo_quiet_nan((int64_t)(p - 1) * n + (q - 1));
}

/* ------------------------------------------------------------------------- */
/* pair enumeration, src/shared/jstep.F90                                    */
/* ------------------------------------------------------------------------- */

/* JSTEP_LEN, src/shared/jstep.F90:124-133 */
int jo_jstep_len(int n, int n_2)
{
  if (!n_2) return (n / 2 > 0) ? n / 2 : 0;
  const int a = (n_2 > 0) ? n_2 : 0;
  return (a < n / 2) ? a : n / 2;
}

static int jo_count_signs(int n, const int *J, int pn[2])
{
  pn[0] = pn[1] = 0;
  for (int i = 0; i < n; ++i) {
    if (J[i] == -1) ++pn[1];
    else if (J[i] == 1) ++pn[0];
    else return -2;
  }
  return 0;
}

/* TRU1 (column-cyclic), src/shared/jstep.F90:9-62 */
int jo_tru1(int n, const int *J, int nn, int *P, int *Q, int pn[2])
{
  pn[0] = pn[1] = 0;
  if (n < 0) return -1;
  if (nn < 0) return -3;
  if (n <= 1) return 0;
  if (jo_count_signs(n, J, pn)) return -2;
  int it = 1, ih = nn;
  for (int iq = 2; iq <= n; ++iq)
    for (int ip = 1; ip < iq; ++ip) {
      if (it > ih) return 0;
      if (J[ip - 1] == J[iq - 1]) { P[it - 1] = ip; Q[it - 1] = iq; ++it; }
      else { P[ih - 1] = ip; Q[ih - 1] = iq; --ih; }
    }
  return it - 1;
}

/* TRU2 (row-cyclic), src/shared/jstep.F90:67-120 */
int jo_tru2(int n, const int *J, int nn, int *P, int *Q, int pn[2])
{
  pn[0] = pn[1] = 0;
  if (n < 0) return -1;
  if (nn < 0) return -3;
  if (n <= 1) return 0;
  if (jo_count_signs(n, J, pn)) return -2;
  int it = 1, ih = nn;
  for (int ip = 1; ip < n; ++ip)
    for (int iq = ip + 1; iq <= n; ++iq) {
      if (it > ih) return 0;
      if (J[ip - 1] == J[iq - 1]) { P[it - 1] = ip; Q[it - 1] = iq; ++it; }
      else { P[ih - 1] = ip; Q[ih - 1] = iq; --ih; }
    }
  return it - 1;
}

/* ------------------------------------------------------------------------- */
/* records, sorting, selection, src/shared/atypes.F90                        */
/* ------------------------------------------------------------------------- */

/* AW_CMP, src/shared/atypes.F90:85-120 */
int jo_aw_cmp(const jo_aw *a, const jo_aw *b)
{
  if (a->w < b->w) return 1;
  if (a->w > b->w) return -1;
  if (a->w == b->w) {
    if (a->b < b->b) return 2;
    if (a->b > b->b) return -2;
    if (a->p < b->p) return 3;
    if (a->p > b->p) return -3;
    if (a->q < b->q) return 4;
    if (a->q > b->q) return -4;
    return 0;
  }
  return (b->w == b->w) ? 5 : -5;
}

/* AW_MERGE, src/shared/atypes.F90:124-176 (0-based offsets i, j, k) */
static int jo_aw_merge(int n, int m, const jo_aw *a, int i, int j, jo_aw *b, int k)
{
  int l = 0, ii = i, jj = j, kk = k;
  const int il = i + n - 1, jl = j + m - 1, kl = k + n + m - 1;
  while (kk <= kl) {
    if (ii > il) { while (kk <= kl) b[kk++] = a[jj++]; break; }
    if (jj > jl) { while (kk <= kl) b[kk++] = a[ii++]; break; }
    const int ll = jo_aw_cmp(&a[ii], &a[jj]);
    if (ll < 0) b[kk] = a[ii++];
    else if (ll == 0) { b[kk] = a[ii++]; ++kk; b[kk] = a[jj++]; }
    else { b[kk] = a[jj++]; ++l; }
    ++kk;
  }
  return l;
}

/* AW_SORT (bottom-up merge sort, A -> B -> A ...), src/shared/atypes.F90:180-214 */
static void jo_aw_sort(int n, jo_aw *a, jo_aw *b)
{
  int w = 1;
  bool d = false;
  while (w < n) {
    const int m = w, w2 = w * 2;
    for (int i = 0; i < n; i += w2) {
      const int j = i + m;
      const int ni = jo_imin(m, n - i), nj = (jo_imin(m, n - j) > 0) ? jo_imin(m, n - j) : 0;
      if (d) jo_aw_merge(ni, nj, b, i, j, a, i);
      else jo_aw_merge(ni, nj, a, i, j, b, i);
    }
    w = w2;
    d = !d;
  }
  if (d)
    memcpy(a, b, (size_t)n * sizeof(jo_aw));
}

/* AW_SRT1 (Baudet-Stevenson odd-even merge-split sort), src/shared/atypes.F90:218-324 */
int jo_aw_srt1(int nn, int nm, jo_aw *dz, int nt)
{
  if (nn < 0) return -1;
  if (nm < nn) return -2;
  if (!nn) return 0;
  if (nt < 1) nt = 1;
  int i = nn % nt;
  if (i > 0) i = nt - i;
  const int epa = nn + i, ept = epa / nt;
  if (2 * epa > nm) return -2;
  for (int k = nn; k < epa; ++k) {
    dz[k].w = jo_quiet_nan(k + 1);
    dz[k].p = dz[k].q = dz[k].b = dz[k].i = 0;
  }
#pragma omp parallel for num_threads(nt) schedule(static, 1)
  for (int t = 0; t < nt; ++t)
    jo_aw_sort(ept, dz + (long)t * ept, dz + (long)t * ept + epa);
  for (;;) {
    int te = 0, l = 0;
#pragma omp parallel for num_threads(nt) schedule(static, 1) reduction(+:l)
    for (int t = 0; t < nt; ++t) {
      if (!(t % 2)) {
        const int ii = t * ept, jj = ii + ept, kk = ii + epa;
        const int m = jo_imin(ept, epa - jj);
        l += jo_aw_merge(ept, (m > 0) ? m : 0, dz, ii, jj, dz, kk);
      }
    }
    te += l;
    l = 0;
#pragma omp parallel for num_threads(nt) schedule(static, 1) reduction(+:l)
    for (int t = 0; t < nt; ++t) {
      const int kk = t * ept, ii = kk + epa;
      if (t % 2) {
        const int jj = ii + ept;
        const int m = jo_imin(ept, 2 * epa - jj);
        l += jo_aw_merge(ept, (m > 0) ? m : 0, dz, ii, jj, dz, kk);
      }
      else if (!t)
        memcpy(dz + kk, dz + ii, (size_t)ept * sizeof(jo_aw));
    }
    te += l;
    if (!te) break;
  }
  return 0;
}

/* AW_SRT2, src/shared/atypes.F90:328-355 */
int jo_aw_srt2(int nn, int nm, jo_aw *dz)
{
  if (nn < 0) return -1;
  if (nm < nn) return -2;
  if (!nn) return 0;
  jo_aw_sort(nn, dz, dz + nn);
  return 0;
}

/* AW_NCP1 (NaN-marking greedy), src/shared/atypes.F90:359-426; step is 1-based into dz */
int jo_aw_ncp1(int n, int nn, int nm, jo_aw *dz, int n_2, int *sl, int *step, int nt)
{
  *sl = 0;
  if (n < 0) return -1;
  if (nn < 0) return -2;
  if (nm < nn) return -3;
  if (n_2 < 0) return -5;
  if (!n || !nn || !n_2) return 0;
  if (nt < 1) nt = 1;
  int i = 1;
  while (*sl < n_2) {
    ++*sl;
    step[*sl - 1] = i;
    if (*sl >= n_2) break;
    const int ap = dz[i - 1].p, aq = dz[i - 1].q;
    int k = nn + 1;
#pragma omp parallel for num_threads(nt) reduction(min:k)
    for (int j = i + 1; j <= nn; ++j) {
      if (dz[j - 1].w == dz[j - 1].w) {
        const int bp = dz[j - 1].p, bq = dz[j - 1].q;
        if ((ap == bp) || (ap == bq) || (aq == bp) || (aq == bq)) dz[j - 1].w = jo_quiet_nan(j);
        else if (j < k) k = j;
      }
    }
    if (k > nn) break;
    i = k;
  }
  return 0;
}

/* AW_NCP2 (bitmap greedy), src/shared/atypes.F90:430-484 */
int jo_aw_ncp2(int n, int nn, int nm, jo_aw *dz, int n_2, int *sl, int *step)
{
  *sl = 0;
  if (n < 0) return -1;
  if (nn < 0) return -2;
  if (nm < nn) return -3;
  if (n_2 < 0) return -5;
  if (!n || !nn || !n_2) return 0;
  bool *r = (bool*)calloc((size_t)n + 1u, sizeof(bool));
  if (!r) return -4;
  int j = 1;
  for (int i = 1; i <= n_2; ++i) {
    step[i - 1] = j;
    r[dz[j - 1].p] = true;
    r[dz[j - 1].q] = true;
    ++j;
    while (j <= nn) {
      if ((dz[j - 1].w == dz[j - 1].w) && !r[dz[j - 1].p] && !r[dz[j - 1].q]) break;
      ++j;
    }
    *sl = i;
    if (j > nn) break;
  }
  free(r);
  return 0;
}

/* AW_NCPT + AW_NCP3 (best greedy over all start offsets), src/shared/atypes.F90:488-592 */
int jo_aw_ncp3(int n, int nn, int nm, jo_aw *dz, int n_2, int *sl, int *step, int nt)
{
  *sl = 0;
  if (n < 0) return -1;
  if (nn < 0) return -2;
  if (nm < nn) return -3;
  if (n_2 < 0) return -5;
  if (!n || !nn || !n_2) return 0;
  if (nt < 1) nt = 1;
  double bw = jo_quiet_nan(n_2);
  int bk = nn + 1;
#pragma omp parallel num_threads(nt)
  {
    int *stp = (int*)malloc((size_t)n_2 * sizeof(int));
#pragma omp for schedule(dynamic, 1)
    for (int i = 1; i <= nn; ++i) {
      const int j = i - 1;
      int mysl = 0;
      if (!stp) continue;
      /* AW_NCP2 on DZ(I:NN) reads only the weights, P and Q */
      jo_aw_ncp2(n, nn - j, nm - j, dz + j, n_2, &mysl, stp);
      if (mysl >= 1) {
        int l = 0;
        for (int k = mysl; k >= 1; --k)
          if (dz[j + stp[k - 1] - 1].w > 0.0) { l = k; break; }
        double mywp = 0.0, mywn = 0.0;
        for (int k = l; k >= 1; --k) mywp = mywp + dz[j + stp[k - 1] - 1].w;
        for (int k = l + 1; k <= mysl; ++k) mywn = mywn + dz[j + stp[k - 1] - 1].w;
        const double myw = mywp + mywn;
        const int ll = j + 1;
#pragma omp critical
        {
          if (!(myw <= bw) || ((myw == bw) && (ll < bk))) {
            *sl = mysl;
            for (int k = 0; k < mysl; ++k) step[k] = stp[k] + j;
            bw = myw;
            bk = ll;
          }
        }
      }
    }
    free(stp);
  }
  return 0;
}

/* ------------------------------------------------------------------------- */
/* the real step engine, src/D/dstep.F90                                     */
/* ------------------------------------------------------------------------- */

typedef int (*jo_tru_fn)(int, const int*, int, int*, int*, int[2]);

/* NaN records to the tail (src/D/dstep.F90:223-245); the sort is a total order
 * on distinct pairs, so any partition gives the same sorted prefix. */
static void jo_partition(int nn, jo_aw *dz)
{
  int i = 0, ii = nn - 1;
  while (i < ii) {
    while ((ii > i) && !(dz[ii].w == dz[ii].w)) --ii;
    while (i < ii) {
      if (dz[i].w == dz[i].w) ++i;
      else { const jo_aw x = dz[i]; dz[i] = dz[ii]; dz[ii] = x; --ii; ++i; break; }
    }
  }
}

/* sort + NCP on the first it records, src/D/dstep.F90:249-265; returns 0 or < 0 */
static int jo_sort_select(int n, int it, int nm, jo_aw *dz, int n_2, int id_ncp, int nt, int *sl, int *step)
{
  int id = (nt > 1) ? jo_aw_srt1(it, nm, dz, nt) : jo_aw_srt2(it, nm, dz);
  if (id < 0) return -11;
  const int ns = jo_imin(it, n_2);
  if (id_ncp == 1) id = jo_aw_ncp1(n, it, nm, dz, ns, sl, step, nt);
  else if (id_ncp == 2) id = jo_aw_ncp2(n, it, nm, dz, ns, sl, step);
  else id = jo_aw_ncp3(n, it, nm, dz, ns, sl, step, nt);
  return (id < 0) ? -13 : 0;
}

/* DSTEP_BUILD, src/D/dstep.F90:138-282 */
static int jo_dstep_build(int n, const double *A, int lda, const int *J, int nn, const int *P, const int *Q,
                          int nm, jo_aw *dz, int tt, int n_2, int id_ncp, int nt, int *sl, int *step)
{
  *sl = 0;
  if (!n || !nn || !n_2) return 0;
  int it = 0, ii = 0;
#pragma omp parallel for num_threads(nt) reduction(+:it)
  for (int i = 1; i <= tt; ++i) {
    jo_aw *r = &dz[i - 1];
    r->p = P[i - 1]; r->q = Q[i - 1]; r->b = r->q - r->p; r->i = i;
    r->w = jo_dmagf2t(n, r->p, r->q, A, lda, J);
    if (r->w == r->w) ++it;
  }
#pragma omp parallel for num_threads(nt) schedule(dynamic, 64) reduction(+:ii)
  for (int i = tt + 1; i <= nn; ++i) {
    jo_aw *r = &dz[i - 1];
    r->p = P[i - 1]; r->q = Q[i - 1]; r->b = r->q - r->p; r->i = i;
    r->w = jo_dmagf2h(n, r->p, r->q, A, lda, J);
    if (r->w < -DBL_MAX) r->w = jo_quiet_nan(i);
    else if (r->w == r->w) ++ii;
  }
  it += ii;
  if (!it) return 0;
  if (it < nn) jo_partition(nn, dz);
  return jo_sort_select(n, it, nm, dz, n_2, id_ncp, nt, sl, step);
}

/* DSTEP_TRANSF, src/D/dstep.F90:286-372.
 * The reference's REDUCTION(MIN:M) over DHSVD2's INFO keeps each thread's last
 * value; here M is the minimum over all pivots (the two agree unless a pivot fails). */
static int jo_dstep_transf(int n, double *U, int ldu, double *A, int lda, double *Z, int ldz, const int *J,
                           double stats[3], jo_aw *dz, int sl, const int *step, double *W, int nt)
{
  int m = INT_MAX;
#pragma omp parallel for num_threads(nt) reduction(min:m)
  for (int i = 0; i < sl; ++i) {
    const int p = dz[step[i] - 1].p, q = dz[step[i] - 1].q;
    double B[4] = { AE(A, lda, p, p), AE(A, lda, q, p), AE(A, lda, p, q), AE(A, lda, q, q) }, V[4];
    const int K[2] = { J[p - 1], J[q - 1] };
    double *Wi = W + 6 * (long)i;
    int info = 0;
    jo_dhsvd2(B, K, V, Wi, JO_TH1FIX, &info);
    dz[step[i] - 1].i = info;
    if (info >= 0) {
      Wi[4] = B[M11];
      Wi[5] = B[M22];
      if (info & 2) {
        jo_dba(V, n, &AE(A, lda, p, 1), &AE(A, lda, q, 1), lda);
        JO_SWAP(V[M21], V[M12]); /* UT2 */
        jo_dab(V, n, &AE(U, ldu, 1, p), &AE(U, ldu, 1, q));
      }
      if (info & 4) jo_dab(Wi, n, &AE(Z, ldz, 1, p), &AE(Z, ldz, 1, q));
    }
    if (info < m) m = info;
  }
  if (m >= 0) {
    m = 0;
#pragma omp parallel for num_threads(nt) reduction(+:m)
    for (int i = 0; i < sl; ++i) {
      const int p = dz[step[i] - 1].p, q = dz[step[i] - 1].q, l = dz[step[i] - 1].i;
      const double *Wi = W + 6 * (long)i;
      if (l & 4) jo_dab(Wi, n, &AE(A, lda, 1, p), &AE(A, lda, 1, q));
      if ((l & 1) && ((l & 2) || (l & 4))) ++m;
      if (!(l & 8)) {
        AE(A, lda, p, p) = Wi[4]; AE(A, lda, q, p) = 0.0; AE(A, lda, p, q) = 0.0; AE(A, lda, q, q) = Wi[5];
      }
    }
  }
  double tw = -0.0;
  int pt = 0, qh = 0;
  if (m >= 0)
    for (int i = 0; i < sl; ++i) {
      const int l = dz[step[i] - 1].i;
      if ((l & 2) || (l & 4)) {
        tw = tw + dz[step[i] - 1].w;
        if (J[dz[step[i] - 1].p - 1] == J[dz[step[i] - 1].q - 1]) ++pt; else ++qh;
      }
    }
  stats[0] = tw; stats[1] = pt; stats[2] = qh;
  return m;
}

static void jo_trace_step(jo_trace *tr, int sl, int nl, const double st[3], const jo_aw *dz, const int *step)
{
  if (!tr) return;
  const int s = tr->n_steps;
  if (s < tr->max_steps) {
    if (tr->sl) tr->sl[s] = sl;
    if (tr->nl) tr->nl[s] = nl;
    if (tr->tw) tr->tw[s] = st ? st[0] : -0.0;
    if (tr->trig) tr->trig[s] = st ? (int)st[1] : 0;
    if (tr->hyp) tr->hyp[s] = st ? (int)st[2] : 0;
  }
  if (tr->piv)
    for (int i = 0; i < sl; ++i)
      if (tr->n_piv < tr->max_piv) {
        tr->piv[2 * tr->n_piv + 0] = dz[step[i] - 1].p;
        tr->piv[2 * tr->n_piv + 1] = dz[step[i] - 1].q;
        ++tr->n_piv;
      }
  ++tr->n_steps;
}

/* optional stop after a number of steps (tests and experiments only; 0 = none) */
static int jo_max_steps = 0;
void jo_set_max_steps(int m) { jo_max_steps = (m > 0) ? m : 0; }
int jo_get_max_steps(void) { return jo_max_steps; }

/* DSTEP_LOOP (with DSTEP_EXEC and JZTJ), src/D/dstep.F90:376-604 */
int jo_dstep_loop(int n, double *U, int ldu, double *A, int lda, double *Z, int ldz,
                  const int *J, double *sigma, int n_2, int id_ncp, int id_tru, int nt, jo_trace *tr)
{
  if (n < 3) return -1;
  if (ldu < n) return -3;
  if (lda < n) return -5;
  if (ldz < n) return -7;
  if (n_2 < 0) return -16;
  if (id_ncp < 0 || id_ncp > 3) return -21;
  if (id_tru < 0 || id_tru > 2) return -22;
  if (nt < 1) nt = 1;
  if (!id_ncp) id_ncp = (nt > 1) ? 1 : 2;
  n_2 = jo_jstep_len(n, n_2);

  const int nn = (n * (n - 1)) / 2;
  int pad = nn % nt;
  if (pad > 0) pad = nt - pad;
  const int nm = 2 * (nn + pad);
  int *P = (int*)malloc((size_t)nn * sizeof(int)), *Q = (int*)malloc((size_t)nn * sizeof(int));
  int *step = (int*)malloc((size_t)(n_2 + 1) * sizeof(int));
  jo_aw *dz = (jo_aw*)malloc((size_t)nm * sizeof(jo_aw));
  double *W = (double*)malloc((size_t)(n_2 + 1) * 6u * sizeof(double));
  int info = 0, pn[2];
  if (!P || !Q || !step || !dz || !W) { info = -20; goto done; }

  const int tt = ((id_tru == 2) ? jo_tru2 : jo_tru1)(n, J, nn, P, Q, pn);
  if (tt < 0) { info = -23; goto done; }
  if (tr) { tr->n_piv = 0; tr->n_steps = 0; }

  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      AE(U, ldu, i + 1, j + 1) = (i == j) ? 1.0 : 0.0;
      AE(Z, ldz, i + 1, j + 1) = (i == j) ? 1.0 : 0.0;
    }

  int s = 0, sl = 0;
  for (;;) {
    double st[3] = { -0.0, 0.0, 0.0 };
    sl = 0;
    const int ib = jo_dstep_build(n, A, lda, J, nn, P, Q, nm, dz, tt, n_2, id_ncp, nt, &sl, step);
    info = (ib < 0) ? ib : 0;
    if (sl <= 0 || info < 0) { jo_trace_step(tr, (info < 0) ? info : sl, -1, NULL, dz, step); break; }
    const int nl = jo_dstep_transf(n, U, ldu, A, lda, Z, ldz, J, st, dz, sl, step, W, nt);
    jo_trace_step(tr, sl, nl, st, dz, step);
    sl = (sl < nl) ? sl : nl;
    if (sl <= 0) break;
    ++s;
    if (jo_max_steps && s >= jo_max_steps) break;
  }
  if (sl < 0) info = sl;
  else if (info >= 0) info = s;

  for (int i = 0; i < n; ++i) {
    sigma[i] = AE(A, lda, i + 1, i + 1);
    AE(A, lda, i + 1, i + 1) = 0.0;
  }
  for (int k = 0; k < nn; ++k) { /* JZTJ, src/D/dstep.F90:447-468 */
    const int ip = P[k], iq = Q[k];
    const double t = AE(Z, ldz, ip, iq);
    AE(Z, ldz, ip, iq) = AE(Z, ldz, iq, ip);
    AE(Z, ldz, iq, ip) = t;
    if (J[ip - 1] != J[iq - 1]) { AE(Z, ldz, ip, iq) = -AE(Z, ldz, ip, iq); AE(Z, ldz, iq, ip) = -AE(Z, ldz, iq, ip); }
  }
done:
  free(W); free(dz); free(step); free(Q); free(P);
  return info;
}

/* One build's weights in record order (TRU1/TRU2), for kernel-level parity tests. */
int jo_dweights(int n, const double *A, int lda, const int *J, int id_tru, int nt, double *w, int *P, int *Q)
{
  const int nn = (n * (n - 1)) / 2;
  int pn[2];
  const int tt = ((id_tru == 2) ? jo_tru2 : jo_tru1)(n, J, nn, P, Q, pn);
  if (tt < 0) return tt;
  if (nt < 1) nt = 1;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 64)
  for (int i = 1; i <= nn; ++i) {
    double x;
    if (i <= tt) x = jo_dmagf2t(n, P[i - 1], Q[i - 1], A, lda, J);
    else {
      x = jo_dmagf2h(n, P[i - 1], Q[i - 1], A, lda, J);
      if (x < -DBL_MAX) x = jo_quiet_nan(i);
    }
    w[i - 1] = x;
  }
  return tt;
}

/* Sort + NCP from given weights (one DSTEP_BUILD without the weight phase). */
int jo_select(int n, int nn, const double *w, const int *P, const int *Q, int n_2, int id_ncp, int nt, int *piv)
{
  if (nt < 1) nt = 1;
  if (!id_ncp) id_ncp = (nt > 1) ? 1 : 2;
  int pad = nn % nt;
  if (pad > 0) pad = nt - pad;
  const int nm = 2 * (nn + pad);
  jo_aw *dz = (jo_aw*)malloc((size_t)(nm + 1) * sizeof(jo_aw));
  int *step = (int*)malloc((size_t)(n_2 + 1) * sizeof(int));
  int sl = 0, it = 0, ret;
  if (!dz || !step) { free(dz); free(step); return -20; }
  for (int i = 0; i < nn; ++i) {
    dz[i].w = w[i]; dz[i].p = P[i]; dz[i].q = Q[i]; dz[i].b = Q[i] - P[i]; dz[i].i = i + 1;
    if (w[i] == w[i]) ++it;
  }
  if (!it || !n_2) { free(dz); free(step); return 0; }
  if (it < nn) jo_partition(nn, dz);
  ret = jo_sort_select(n, it, nm, dz, n_2, id_ncp, nt, &sl, step);
  if (!ret)
    for (int i = 0; i < sl; ++i) { piv[2 * i] = dz[step[i] - 1].p; piv[2 * i + 1] = dz[step[i] - 1].q; }
  free(dz); free(step);
  return ret ? ret : sl;
}

/* entry points shared with the complex engine (jk_oracle_z.c) */
void jo_khsvd2_shared(const double A[4], const int J[2], double G[2], double U[4], double Z[4], int s, double th1, int *info)
{
  jo_khsvd2(A, J, G, U, Z, s, th1, info);
}
int jo_sort_select_shared(int n, int it, int nm, jo_aw *dz, int n_2, int id_ncp, int nt, int *sl, int *step)
{
  return jo_sort_select(n, it, nm, dz, n_2, id_ncp, nt, sl, step);
}
void jo_partition_shared(int nn, jo_aw *dz) { jo_partition(nn, dz); }
void jo_trace_step_shared(jo_trace *tr, int sl, int nl, const double st[3], const jo_aw *dz, const int *step)
{
  jo_trace_step(tr, sl, nl, st, dz, step);
}
