/*
 * jk_oracle_z.c -- TEST INFRASTRUCTURE ONLY: CPU restatement of venovako/JKogb's
 * complex step loop (zjk): src/Z/ztransf.F90 and src/Z/zstep.F90.
 * Complex numbers are (re, im) pairs; every complex helper spells out the
 * reference's own fma sequence (ZZFMA, ZZMUL, ...), not C99 complex arithmetic.
 */
#include "jk_oracle_impl.h"

static int jo_zba_quirk = 1;
void jo_set_zba_quirk(int on) { jo_zba_quirk = on ? 1 : 0; }

static inline jo_z jo_conj(jo_z a) { return jo_zc(a.re, -a.im); }
static inline jo_z jo_zneg(jo_z a) { return jo_zc(-a.re, -a.im); }
static inline bool jo_zeq0(jo_z a) { return (a.re == 0.0) && (a.im == 0.0); }
static inline bool jo_zne1(jo_z a) { return (a.re != 1.0) || (a.im != 0.0); }
static inline double jo_zabs(jo_z a) { return jo_hypot(a.re, a.im); }

/* ZDFMA, src/Z/ztransf.F90:130-141 */
static inline jo_z jo_zdfma(double a, jo_z b, jo_z c) { return jo_zc(fma(a, b.re, c.re), fma(a, b.im, c.im)); }

/* ZZFMA, src/Z/ztransf.F90:162-174 */
static inline jo_z jo_zzfma(jo_z a, jo_z b, jo_z c)
{
  double f = fma(-a.im, b.im, c.re);
  const double r = fma(a.re, b.re, f);
  f = fma(a.im, b.re, c.im);
  return jo_zc(r, fma(a.re, b.im, f));
}

/* ZZMUL, src/Z/ztransf.F90:193-205 */
static inline jo_z jo_zzmul(jo_z a, jo_z b)
{
  double f = a.im * b.im;
  const double r = fma(a.re, b.re, -f);
  f = a.im * b.re;
  return jo_zc(r, fma(a.re, b.im, f));
}

/* ZDDIV, src/Z/ztransf.F90:209-215 */
static inline jo_z jo_zddiv(jo_z a, double b) { return jo_zc(a.re / b, a.im / b); }

/* ZZDIV, src/Z/ztransf.F90:220-227 */
static inline jo_z jo_zzdiv(jo_z a, jo_z b)
{
  const double f = jo_zabs(b);
  return jo_zddiv(jo_zzmul(jo_conj(jo_zddiv(b, f)), a), f);
}

/* the ratio of BA/AB/ABODNZF2: ZDDIV when the divisor is real, else ZZDIV */
static inline jo_z jo_zratio(jo_z num, jo_z den)
{
  return (den.im == 0.0) ? jo_zddiv(num, den.re) : jo_zzdiv(num, den);
}

/* C1A, src/Z/ztransf.F90:231-241 */
static void jo_zc1a(const double B[4], jo_z *a1, jo_z *a2)
{
  const jo_z c1 = jo_zddiv(jo_zdfma(B[M12], *a2, *a1), B[M11]);
  const jo_z c2 = jo_zddiv(jo_zdfma(B[M21], *a1, *a2), B[M22]);
  *a1 = c1; *a2 = c2;
}

/* C2A, src/Z/ztransf.F90:245-258 */
static void jo_zc2a(const double B[4], jo_z A[4])
{
  jo_z C[4];
  for (int j = 0; j < 2; ++j) {
    C[2 * j + 0] = jo_zddiv(jo_zdfma(B[M12], A[2 * j + 1], A[2 * j + 0]), B[M11]);
    C[2 * j + 1] = jo_zddiv(jo_zdfma(B[M21], A[2 * j + 0], A[2 * j + 1]), B[M22]);
  }
  memcpy(A, C, sizeof(C));
}

/* A2C, src/Z/ztransf.F90:262-275 */
static void jo_za2c(jo_z A[4], const double B[4])
{
  jo_z C[4];
  for (int i = 0; i < 2; ++i) {
    C[i + 0] = jo_zddiv(jo_zdfma(B[M21], A[i + 2], A[i + 0]), B[M11]);
    C[i + 2] = jo_zddiv(jo_zdfma(B[M12], A[i + 0], A[i + 2]), B[M22]);
  }
  memcpy(A, C, sizeof(C));
}

/* ZPOLAR, src/Z/ztransf.F90:112-126 */
static void jo_zpolar(jo_z z, double *a, jo_z *e)
{
  *a = jo_hypot(z.re, z.im);
  const double c = copysign(fmin(fabs(z.re) / *a, 1.0), z.re);
  const double s = z.im / fmax(*a, JO_MINF);
  *e = jo_zc(c, s);
}

#define JO_ZSWAP(a, b) do { const jo_z t_ = (a); (a) = (b); (b) = t_; } while (0)

/* ZHSVD2T, src/Z/ztransf.F90:641-835 */
static void jo_zhsvd2t(jo_z A[4], const int J[2], jo_z U[4], jo_z Z[4], int *info)
{
  double Q[4], c, t, w;
  jo_z r, s;
  bool p, d = true;

  if (jo_zeq0(A[M21])) c = jo_zabs(A[M11]);
  else if (jo_zeq0(A[M11])) { c = jo_zabs(A[M21]); d = false; }
  else { c = jo_hypot(jo_zabs(A[M11]), jo_zabs(A[M21])); d = false; }
  if (jo_zeq0(A[M12])) t = jo_zabs(A[M22]);
  else if (jo_zeq0(A[M22])) { t = jo_zabs(A[M12]); d = false; }
  else { t = jo_hypot(jo_zabs(A[M12]), jo_zabs(A[M22])); d = false; }

  if (c < t) {
    JO_ZSWAP(A[M11], A[M12]); JO_ZSWAP(A[M21], A[M22]);
    if (J[0] == J[1]) { JO_ZSWAP(Z[M11], Z[M12]); JO_ZSWAP(Z[M21], Z[M22]); }
    p = true;
    w = t;
  }
  else { p = false; w = c; }

  jo_zpolar(A[M11], &c, &r);
  if (jo_zne1(r)) {
    s = jo_conj(r);
    U[M11] = jo_zzmul(U[M11], s); U[M12] = jo_zzmul(U[M12], s);
    A[M11] = jo_zzmul(A[M11], s); A[M12] = jo_zzmul(A[M12], s);
  }
  jo_zpolar(A[M21], &t, &s);
  if (jo_zne1(s)) {
    r = jo_conj(s);
    U[M21] = jo_zzmul(U[M21], r); U[M22] = jo_zzmul(U[M22], r);
    A[M21] = jo_zzmul(A[M21], r); A[M22] = jo_zzmul(A[M22], r);
  }

  if (A[M11].re < A[M21].re) {
    JO_ZSWAP(U[M11], U[M21]); JO_ZSWAP(U[M12], U[M22]);
    JO_ZSWAP(A[M11], A[M21]); JO_ZSWAP(A[M12], A[M22]);
  }

  if (!d) {
    t = A[M21].re / A[M11].re;
    c = sqrt(fma(t, t, 1.0));
    Q[M11] = c; Q[M21] = -t; Q[M12] = t; Q[M22] = c;
    jo_zc2a(Q, U);
    jo_zc1a(Q, &A[M12], &A[M22]);
  }
  A[M11] = jo_zc(w, 0.0);
  A[M21] = jo_zc(0.0, 0.0);

  if ((J[0] != J[1]) && p) {
    JO_ZSWAP(A[M11], A[M12]); JO_ZSWAP(A[M21], A[M22]);
    JO_ZSWAP(U[M11], U[M21]); JO_ZSWAP(U[M12], U[M22]);
    JO_ZSWAP(A[M11], A[M21]); JO_ZSWAP(A[M12], A[M22]);
    jo_zpolar(A[M21], &t, &s);
    if (jo_zne1(s)) {
      r = jo_conj(s);
      Z[M11] = jo_zzmul(Z[M11], r); Z[M21] = jo_zzmul(Z[M21], r);
      A[M11] = jo_zzmul(A[M11], r); A[M21] = jo_zzmul(A[M21], r);
    }
    jo_zpolar(A[M11], &c, &r);
    if (jo_zne1(r)) {
      s = jo_conj(r);
      U[M11] = jo_zzmul(U[M11], s); U[M12] = jo_zzmul(U[M12], s);
      A[M11] = jo_zzmul(A[M11], s);
    }
  }
  else {
    jo_zpolar(A[M12], &c, &r);
    if (jo_zne1(r)) {
      s = jo_conj(r);
      Z[M12] = jo_zzmul(Z[M12], s); Z[M22] = jo_zzmul(Z[M22], s);
      A[M12] = jo_zzmul(A[M12], s); A[M22] = jo_zzmul(A[M22], s);
    }
    jo_zpolar(A[M22], &t, &s);
    if (jo_zne1(s)) {
      r = jo_conj(s);
      U[M21] = jo_zzmul(U[M21], r); U[M22] = jo_zzmul(U[M22], r);
      A[M22] = jo_zzmul(A[M22], r);
    }
  }
  *info = d ? 0 : 1;
}

/* ZHSVD2S, src/Z/ztransf.F90:839-880 */
static void jo_zhsvd2s(jo_z A[4], const int J[2], jo_z U[4], jo_z Z[4], int *info)
{
  const int t = J[0] + J[1];
  if (((t == 2) && (A[M11].re < A[M22].re)) || ((t == -2) && (A[M22].re < A[M11].re))) {
    A[M21] = U[M11]; A[M12] = U[M12];
    U[M11] = U[M21]; U[M12] = U[M22];
    U[M21] = A[M21]; U[M22] = A[M12];
    A[M21] = A[M11]; A[M11] = A[M22]; A[M22] = A[M21];
    A[M21] = Z[M11]; A[M12] = Z[M21];
    Z[M11] = Z[M12]; Z[M21] = Z[M22];
    Z[M12] = A[M21]; Z[M22] = A[M12];
  }
  if (!(*info & 8)) { A[M21] = jo_zc(0.0, 0.0); A[M12] = jo_zc(0.0, 0.0); }
  if (jo_zne1(U[M11]) || !jo_zeq0(U[M21]) || !jo_zeq0(U[M12]) || jo_zne1(U[M22])) *info += 2;
  if (jo_zne1(Z[M11]) || !jo_zeq0(Z[M21]) || !jo_zeq0(Z[M12]) || jo_zne1(Z[M22])) *info += 4;
}

/* ZSCALEA, src/Z/ztransf.F90:884-921 */
static void jo_zscalea(jo_z A[4], int *s)
{
  *s = INT_MAX;
  for (int j = 0; j < 2; ++j)
    for (int i = 0; i < 2; ++i) {
      double aa = fabs(A[2 * j + i].re);
      if (!(aa <= DBL_MAX)) { *s = -((j + 1) * 2 + (i + 1)); return; }
      *s = jo_imin(*s, JO_EH - jo_exponent(fmax(aa, JO_MINF)) - 2);
      aa = fabs(A[2 * j + i].im);
      if (!(aa <= DBL_MAX)) { *s = -((j + 1) * 2 + (i + 1)); return; }
      *s = jo_imin(*s, JO_EH - jo_exponent(fmax(aa, JO_MINF)) - 2);
    }
  if (*s != 0)
    for (int k = 0; k < 4; ++k)
      A[k] = jo_zc(jo_scale(A[k].re, *s), jo_scale(A[k].im, *s));
}

/* the real triangular kernel KHSVD2 is shared (src/shared/ktransf.F90);
 * jk_oracle.c exposes it through this thin wrapper */
void jo_khsvd2_shared(const double A[4], const int J[2], double G[2], double U[4], double Z[4], int s, double th1, int *info);

/* ZHSVD2 (argument-checking build), src/Z/ztransf.F90:925-1009 */
void jo_zhsvd2(jo_z A[4], const int J[2], jo_z U[4], jo_z Z[4], double th1, int *info)
{
  double G[2] = { 0.0, 0.0 }, W[4] = { 0.0, 0.0, 0.0, 0.0 }, B[4] = { 0.0, 0.0, 0.0, 0.0 }, C[4] = { 0.0, 0.0, 0.0, 0.0 };
  int s;

  if (abs(J[0]) != 1) *info = -1;
  else if (abs(J[1]) != 1) *info = -2;
  else *info = 0;
  if (*info) return;

  jo_zscalea(A, &s);
  if (s <= -3) { *info = s; return; }

  U[M11] = jo_zc(1.0, 0.0); U[M21] = jo_zc(0.0, 0.0); U[M12] = jo_zc(0.0, 0.0); U[M22] = jo_zc(1.0, 0.0);
  Z[M11] = jo_zc(1.0, 0.0); Z[M21] = jo_zc(0.0, 0.0); Z[M12] = jo_zc(0.0, 0.0); Z[M22] = jo_zc(1.0, 0.0);

  jo_zhsvd2t(A, J, U, Z, info);
  if (*info > 0) {
    W[M11] = A[M11].re; W[M21] = A[M21].re; W[M12] = A[M12].re; W[M22] = A[M22].re;
    jo_khsvd2_shared(W, J, G, B, C, s, th1, info);
  }
  else if (*info == 0) {
    if (s == 0) { W[M11] = A[M11].re; W[M22] = A[M22].re; }
    else { W[M11] = jo_scale(A[M11].re, -s); W[M22] = jo_scale(A[M22].re, -s); }
  }
  if (*info < 0) return;
  if (*info > 0) {
    jo_zc2a(B, U);
    jo_za2c(Z, C);
    if (!(*info & 8)) { W[M11] = G[0]; W[M22] = G[1]; }
    else {
      if (s != 0)
        for (int k = 0; k < 4; ++k)
          A[k] = jo_zc(jo_scale(A[k].re, -s), jo_scale(A[k].im, -s));
      jo_zc2a(B, A);
      jo_za2c(A, C);
      goto l2;
    }
  }
  A[M11] = jo_zc(W[M11], 0.0);
  A[M22] = jo_zc(W[M22], 0.0);
l2:
  jo_zhsvd2s(A, J, U, Z, info);
}

/* BA, src/Z/ztransf.F90:279-365 (with the branch at :325 as a switch) */
void jo_zba(const jo_z B[4], int n, jo_z *x, jo_z *y, int lda)
{
  jo_z r1, r2, xx, yy;
  long i = 0;
  if (jo_zabs(B[M11]) >= jo_zabs(B[M12])) {
    r1 = jo_zratio(B[M12], B[M11]);
    if (jo_zabs(B[M22]) >= jo_zabs(B[M21])) {
      r2 = jo_zratio(B[M21], B[M22]);
      for (int j = 0; j < n; ++j, i += lda) {
        xx = jo_zzfma(r1, y[i], x[i]); yy = jo_zzfma(r2, x[i], y[i]);
        x[i] = jo_zzmul(xx, B[M11]); y[i] = jo_zzmul(yy, B[M22]);
      }
    }
    else {
      r2 = jo_zratio(B[M22], B[M21]);
      const jo_z rr = jo_zba_quirk ? r1 : r2;
      for (int j = 0; j < n; ++j, i += lda) {
        xx = jo_zzfma(r1, y[i], x[i]); yy = jo_zzfma(rr, y[i], x[i]);
        x[i] = jo_zzmul(xx, B[M11]); y[i] = jo_zzmul(yy, B[M21]);
      }
    }
  }
  else {
    r1 = jo_zratio(B[M11], B[M12]);
    if (jo_zabs(B[M22]) >= jo_zabs(B[M21])) {
      r2 = jo_zratio(B[M21], B[M22]);
      for (int j = 0; j < n; ++j, i += lda) {
        xx = jo_zzfma(r1, x[i], y[i]); yy = jo_zzfma(r2, x[i], y[i]);
        x[i] = jo_zzmul(xx, B[M12]); y[i] = jo_zzmul(yy, B[M22]);
      }
    }
    else {
      r2 = jo_zratio(B[M22], B[M21]);
      for (int j = 0; j < n; ++j, i += lda) {
        xx = jo_zzfma(r1, x[i], y[i]); yy = jo_zzfma(r2, y[i], x[i]);
        x[i] = jo_zzmul(xx, B[M12]); y[i] = jo_zzmul(yy, B[M21]);
      }
    }
  }
}

/* AB, src/Z/ztransf.F90:369-448 */
void jo_zab(const jo_z B[4], int m, jo_z *x, jo_z *y)
{
  jo_z r1, r2, xx, yy;
  if (jo_zabs(B[M11]) >= jo_zabs(B[M21])) {
    r1 = jo_zratio(B[M21], B[M11]);
    if (jo_zabs(B[M22]) >= jo_zabs(B[M12])) {
      r2 = jo_zratio(B[M12], B[M22]);
      for (int i = 0; i < m; ++i) {
        xx = jo_zzfma(y[i], r1, x[i]); yy = jo_zzfma(x[i], r2, y[i]);
        x[i] = jo_zzmul(xx, B[M11]); y[i] = jo_zzmul(yy, B[M22]);
      }
    }
    else {
      r2 = jo_zratio(B[M22], B[M12]);
      for (int i = 0; i < m; ++i) {
        xx = jo_zzfma(y[i], r1, x[i]); yy = jo_zzfma(y[i], r2, x[i]);
        x[i] = jo_zzmul(xx, B[M11]); y[i] = jo_zzmul(yy, B[M12]);
      }
    }
  }
  else {
    r1 = jo_zratio(B[M11], B[M21]);
    if (jo_zabs(B[M22]) >= jo_zabs(B[M12])) {
      r2 = jo_zratio(B[M12], B[M22]);
      for (int i = 0; i < m; ++i) {
        xx = jo_zzfma(x[i], r1, y[i]); yy = jo_zzfma(x[i], r2, y[i]);
        x[i] = jo_zzmul(xx, B[M21]); y[i] = jo_zzmul(yy, B[M22]);
      }
    }
    else {
      r2 = jo_zratio(B[M22], B[M12]);
      for (int i = 0; i < m; ++i) {
        xx = jo_zzfma(x[i], r1, y[i]); yy = jo_zzfma(y[i], r2, x[i]);
        x[i] = jo_zzmul(xx, B[M21]); y[i] = jo_zzmul(yy, B[M12]);
      }
    }
  }
}

/* ABODNZF2, src/Z/ztransf.F90:452-637 (p, q 1-based; rows p and q skipped) */
double jo_abodnzf2(const jo_z B[4], int m, const jo_z *x, const jo_z *y, jo_z aqp, jo_z apq, int p, int q)
{
  double d = 0.0, axi, ayi, axx, ayy;
  axi = x[q - 1].re; ayi = x[q - 1].im; axx = aqp.re; ayy = aqp.im;
  d = fma(axi - axx, axi + axx, d);
  d = fma(ayi - ayy, ayi + ayy, d);
  axi = y[p - 1].re; ayi = y[p - 1].im; axx = apq.re; ayy = apq.im;
  d = fma(axi - axx, axi + axx, d);
  d = fma(ayi - ayy, ayi + ayy, d);

  const int c1 = (jo_zabs(B[M11]) >= jo_zabs(B[M21]));
  const jo_z r1 = c1 ? jo_zratio(B[M21], B[M11]) : jo_zratio(B[M11], B[M21]);
  const int c2 = (jo_zabs(B[M22]) >= jo_zabs(B[M12]));
  const jo_z r2 = c2 ? jo_zratio(B[M12], B[M22]) : jo_zratio(B[M22], B[M12]);
  for (int i = 0; i < m; ++i) {
    jo_z xx, yy;
    if ((i == p - 1) || (i == q - 1))
      continue;
    if (c1) xx = jo_zzmul(jo_zzfma(y[i], r1, x[i]), B[M11]);
    else xx = jo_zzmul(jo_zzfma(x[i], r1, y[i]), B[M21]);
    if (c2) yy = jo_zzmul(jo_zzfma(x[i], r2, y[i]), B[M22]);
    else yy = jo_zzmul(jo_zzfma(y[i], r2, x[i]), B[M12]);
    axi = jo_zabs(x[i]);
    axx = jo_zabs(xx);
    ayi = jo_zabs(y[i]);
    ayy = jo_zabs(yy);
    d = fma((axi - axx), (axi + axx), d);
    d = fma((ayi - ayy), (ayi + ayy), d);
  }
  return d;
}

#define ZE(A, lda, i, j) ((A)[(long)((j) - 1) * (lda) + ((i) - 1)])

/* ZMAGF2T, src/Z/zstep.F90:12-39 */
double jo_zmagf2t(int n, int p, int q, const jo_z *A, int lda, const int *J)
{
  const jo_z app = ZE(A, lda, p, p), aqp = ZE(A, lda, q, p), apq = ZE(A, lda, p, q), aqq = ZE(A, lda, q, q);
  const bool nz = !jo_zeq0(aqp) || !jo_zeq0(apq) || (app.im != 0.0) || (aqq.im != 0.0) || jo_neg(app.re) || jo_neg(aqq.re);
  switch (J[p - 1] + J[q - 1]) {
  case -2:
    if (nz || (aqq.re < app.re)) return jo_dasum4(aqp.re, aqp.im, apq.re, apq.im);
    return jo_quiet_nan((int64_t)(p - 1) * n + (q - 1));
  case 2:
    if (nz || (app.re < aqq.re)) return jo_dasum4(aqp.re, aqp.im, apq.re, apq.im);
    return jo_quiet_nan((int64_t)(p - 1) * n + (q - 1));
  default:
    return jo_quiet_nan((int64_t)(p - 1) * n + (q - 1));
  }
}

/* ZMAGF2H, src/Z/zstep.F90:43-74 */
double jo_zmagf2h(int n, int p, int q, const jo_z *A, int lda, const int *J)
{
  const jo_z app = ZE(A, lda, p, p), aqp = ZE(A, lda, q, p), apq = ZE(A, lda, p, q), aqq = ZE(A, lda, q, q);
  if (!jo_zeq0(aqp) || !jo_zeq0(apq) || (app.im != 0.0) || (aqq.im != 0.0) || jo_neg(app.re) || jo_neg(aqq.re)) {
    jo_z A2[4] = { app, aqp, apq, aqq }, U2[4], Z2[4];
    const int J2[2] = { J[p - 1], J[q - 1] };
    int info = 0;
    jo_zhsvd2(A2, J2, U2, Z2, JO_TH1FIX, &info);
    if (info < 0) return jo_quiet_nan((int64_t)(p - 1) * n + (q - 1));
    if (!(info & 1)) return 0.0;
    if (!(info & 4)) return jo_dasum4(aqp.re, aqp.im, apq.re, apq.im);
    if (!(info & 8))
      return jo_abodnzf2(Z2, n, &ZE(A, lda, 1, p), &ZE(A, lda, 1, q), jo_zc(0.0, 0.0), jo_zc(0.0, 0.0), p, q);
    return jo_abodnzf2(Z2, n, &ZE(A, lda, 1, p), &ZE(A, lda, 1, q), A2[M21], A2[M12], p, q);
  }
  return jo_quiet_nan((int64_t)(p - 1) * n + (q - 1));
}

/* sort + select and the partition are shared with the real engine */
int jo_sort_select_shared(int n, int it, int nm, jo_aw *dz, int n_2, int id_ncp, int nt, int *sl, int *step);
void jo_partition_shared(int nn, jo_aw *dz);

/* ZSTEP_BUILD, src/Z/zstep.F90:140-284 */
static int jo_zstep_build(int n, const jo_z *A, int lda, const int *J, int nn, const int *P, const int *Q,
                          int nm, jo_aw *dz, int tt, int n_2, int id_ncp, int nt, int *sl, int *step)
{
  *sl = 0;
  if (!n || !nn || !n_2) return 0;
  int it = 0, ii = 0;
#pragma omp parallel for num_threads(nt) reduction(+:it)
  for (int i = 1; i <= tt; ++i) {
    jo_aw *r = &dz[i - 1];
    r->p = P[i - 1]; r->q = Q[i - 1]; r->b = r->q - r->p; r->i = i;
    r->w = jo_zmagf2t(n, r->p, r->q, A, lda, J);
    if (r->w == r->w) ++it;
  }
#pragma omp parallel for num_threads(nt) schedule(dynamic, 64) reduction(+:ii)
  for (int i = tt + 1; i <= nn; ++i) {
    jo_aw *r = &dz[i - 1];
    r->p = P[i - 1]; r->q = Q[i - 1]; r->b = r->q - r->p; r->i = i;
    r->w = jo_zmagf2h(n, r->p, r->q, A, lda, J);
    if (r->w < -DBL_MAX) r->w = jo_quiet_nan(i);
    else if (r->w == r->w) ++ii;
  }
  it += ii;
  if (!it) return 0;
  if (it < nn) jo_partition_shared(nn, dz);
  return jo_sort_select_shared(n, it, nm, dz, n_2, id_ncp, nt, sl, step);
}

/* ZSTEP_TRANSF, src/Z/zstep.F90:288-375 (M = min over all pivots, as in the real engine) */
static int jo_zstep_transf(int n, jo_z *U, int ldu, jo_z *A, int lda, jo_z *Z, int ldz, const int *J,
                           double stats[3], jo_aw *dz, int sl, const int *step, jo_z *W, int nt)
{
  int m = INT_MAX;
#pragma omp parallel for num_threads(nt) reduction(min:m)
  for (int i = 0; i < sl; ++i) {
    const int p = dz[step[i] - 1].p, q = dz[step[i] - 1].q;
    jo_z B[4] = { ZE(A, lda, p, p), ZE(A, lda, q, p), ZE(A, lda, p, q), ZE(A, lda, q, q) }, V[4];
    const int K[2] = { J[p - 1], J[q - 1] };
    jo_z *Wi = W + 6 * (long)i;
    int info = 0;
    jo_zhsvd2(B, K, V, Wi, JO_TH1FIX, &info);
    dz[step[i] - 1].i = info;
    if (info >= 0) {
      Wi[4] = jo_zc(B[M11].re, 0.0);
      Wi[5] = jo_zc(B[M22].re, 0.0);
      if (info & 2) {
        jo_zba(V, n, &ZE(A, lda, p, 1), &ZE(A, lda, q, 1), lda);
        /* UH2, src/Z/ztransf.F90:79-90 */
        V[M11] = jo_conj(V[M11]);
        const jo_z u21 = V[M21];
        V[M21] = jo_conj(V[M12]);
        V[M12] = jo_conj(u21);
        V[M22] = jo_conj(V[M22]);
        jo_zab(V, n, &ZE(U, ldu, 1, p), &ZE(U, ldu, 1, q));
      }
      if (info & 4) jo_zab(Wi, n, &ZE(Z, ldz, 1, p), &ZE(Z, ldz, 1, q));
    }
    if (info < m) m = info;
  }
  if (m >= 0) {
    m = 0;
#pragma omp parallel for num_threads(nt) reduction(+:m)
    for (int i = 0; i < sl; ++i) {
      const int p = dz[step[i] - 1].p, q = dz[step[i] - 1].q, l = dz[step[i] - 1].i;
      const jo_z *Wi = W + 6 * (long)i;
      if (l & 4) jo_zab(Wi, n, &ZE(A, lda, 1, p), &ZE(A, lda, 1, q));
      if ((l & 1) && ((l & 2) || (l & 4))) ++m;
      if (!(l & 8)) {
        ZE(A, lda, p, p) = Wi[4]; ZE(A, lda, q, p) = jo_zc(0.0, 0.0);
        ZE(A, lda, p, q) = jo_zc(0.0, 0.0); ZE(A, lda, q, q) = Wi[5];
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

void jo_trace_step_shared(jo_trace *tr, int sl, int nl, const double st[3], const jo_aw *dz, const int *step);
int jo_get_max_steps(void);

/* ZSTEP_LOOP (with ZSTEP_EXEC and JZHJ), src/Z/zstep.F90:379-615 */
int jo_zstep_loop(int n, jo_z *U, int ldu, jo_z *A, int lda, jo_z *Z, int ldz,
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
  jo_z *W = (jo_z*)malloc((size_t)(n_2 + 1) * 6u * sizeof(jo_z));
  int info = 0, pn[2];
  if (!P || !Q || !step || !dz || !W) { info = -20; goto done; }

  const int tt = ((id_tru == 2) ? jo_tru2 : jo_tru1)(n, J, nn, P, Q, pn);
  if (tt < 0) { info = -23; goto done; }
  if (tr) { tr->n_piv = 0; tr->n_steps = 0; }

  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      ZE(U, ldu, i + 1, j + 1) = jo_zc((i == j) ? 1.0 : 0.0, 0.0);
      ZE(Z, ldz, i + 1, j + 1) = jo_zc((i == j) ? 1.0 : 0.0, 0.0);
    }

  int s = 0, sl = 0;
  for (;;) {
    double st[3] = { -0.0, 0.0, 0.0 };
    sl = 0;
    const int ib = jo_zstep_build(n, A, lda, J, nn, P, Q, nm, dz, tt, n_2, id_ncp, nt, &sl, step);
    info = (ib < 0) ? ib : 0;
    if (sl <= 0 || info < 0) { jo_trace_step_shared(tr, (info < 0) ? info : sl, -1, NULL, dz, step); break; }
    const int nl = jo_zstep_transf(n, U, ldu, A, lda, Z, ldz, J, st, dz, sl, step, W, nt);
    jo_trace_step_shared(tr, sl, nl, st, dz, step);
    sl = (sl < nl) ? sl : nl;
    if (sl <= 0) break;
    ++s;
    if (jo_get_max_steps() && s >= jo_get_max_steps()) break;
  }
  if (sl < 0) info = sl;
  else if (info >= 0) info = s;

  for (int i = 0; i < n; ++i) {
    sigma[i] = ZE(A, lda, i + 1, i + 1).re;
    ZE(A, lda, i + 1, i + 1) = jo_zc(0.0, 0.0);
  }
  for (int k = 0; k < nn; ++k) { /* JZHJ, src/Z/zstep.F90:451-478 */
    const int ip = P[k], iq = Q[k];
    const jo_z t = ZE(Z, ldz, ip, iq);
    ZE(Z, ldz, ip, iq) = jo_conj(ZE(Z, ldz, iq, ip));
    ZE(Z, ldz, iq, ip) = jo_conj(t);
    if (J[ip - 1] != J[iq - 1]) { ZE(Z, ldz, ip, iq) = jo_zneg(ZE(Z, ldz, ip, iq)); ZE(Z, ldz, iq, ip) = jo_zneg(ZE(Z, ldz, iq, ip)); }
  }
  for (int i = 1; i <= n; ++i)
    ZE(Z, ldz, i, i) = jo_conj(ZE(Z, ldz, i, i));
done:
  free(W); free(dz); free(step); free(Q); free(P);
  return info;
}

/* One complex build's weights in record order (TRU1/TRU2). */
int jo_zweights(int n, const jo_z *A, int lda, const int *J, int id_tru, int nt, double *w, int *P, int *Q)
{
  const int nn = (n * (n - 1)) / 2;
  int pn[2];
  const int tt = ((id_tru == 2) ? jo_tru2 : jo_tru1)(n, J, nn, P, Q, pn);
  if (tt < 0) return tt;
  if (nt < 1) nt = 1;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 64)
  for (int i = 1; i <= nn; ++i) {
    double x;
    if (i <= tt) x = jo_zmagf2t(n, P[i - 1], Q[i - 1], A, lda, J);
    else {
      x = jo_zmagf2h(n, P[i - 1], Q[i - 1], A, lda, J);
      if (x < -DBL_MAX) x = jo_quiet_nan(i);
    }
    w[i - 1] = x;
  }
  return tt;
}
