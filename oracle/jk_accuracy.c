/*
 * jk_accuracy.c -- TEST INFRASTRUCTURE ONLY: the accuracy oracle.
 *
 * The hyperbolic singular values of a square matrix Y with signature J, computed in
 * extended precision by a method independent of the reference's: the one-sided
 * hyperbolic Jacobi method.  Columns i, j of W = Y (in __float128 or long double) are
 * orthogonalised pair by pair, by a plane rotation when J_i = J_j and by a hyperbolic
 * rotation when J_i != J_j; both keep W V = Y V with V J-orthogonal (V^T J V = J), so
 * at convergence W = U diag(sigma) with U orthogonal and sigma_i = ||W(:,i)||, the
 * hyperbolic singular value attached to J_i.  These are the values the reference's
 * DSTEP_LOOP returns in SIGMA (src/D/dstep.F90:594-602): Y J Y^T has the eigenvalues
 * J_i sigma_i^2, so the multiset of sigma within each sign class is an invariant of Y
 * and J, whichever algorithm finds it.  The column pairs of one sweep are taken in
 * round-robin order (n/2 disjoint pairs per round, in parallel); a sweep with no
 * rotation ends the iteration.
 *
 * Two instantiations: jq_*_q in __float128 (libquadmath; unit roundoff 1e-34) and
 * jq_*_ld in long double (x87 80-bit; unit roundoff 5e-20, much faster), used where
 * __float128 would take too long; the two are cross-checked by the tests.
 * Complex matrices are interleaved (re, im) doubles; their columns are rotated after a
 * phase change that makes the pair's inner product real, which leaves sigma unchanged.
 */
#include <math.h>
#include <quadmath.h>
#include <stdlib.h>
#include <string.h>

#define JQ_DEFINE(SUF, T, SQRT, FABS, U16) /* U16: 16 unit roundoffs of T */                                                                   \
  /* real: returns the sweeps taken (> 0), or -1 if max_sweeps were not enough */                     \
  int jq_dsigma_##SUF(int n, const double *Y, int ldy, const int *J, double *sigma, int nt,            \
                      int max_sweeps)                                                                   \
  {                                                                                                     \
    const int m = n + (n & 1); /* round-robin over an even count, index n is a dummy */                \
    T *W = (T *)malloc(sizeof(T) * (size_t)n * n);                                                      \
    int *pos = (int *)malloc(sizeof(int) * (size_t)m);                                                  \
    if (!W || !pos) { free(W); free(pos); return -2; }                                                  \
    for (int j = 0; j < n; ++j)                                                                         \
      for (int i = 0; i < n; ++i) W[(size_t)j * n + i] = (T)Y[(size_t)j * ldy + i];                     \
    const T tol = (T)n * (T)(U16);                                                                      \
    int sweep = 0, done = 0;                                                                            \
    while (!done && sweep < max_sweeps) {                                                               \
      ++sweep;                                                                                          \
      int rotated = 0;                                                                                  \
      for (int k = 0; k < m; ++k) pos[k] = k;                                                           \
      for (int r = 0; r < m - 1; ++r) {                                                                 \
        _Pragma("omp parallel for num_threads(nt) schedule(dynamic, 1) reduction(+ : rotated)")         \
        for (int h = 0; h < m / 2; ++h) {                                                               \
          int i = pos[h], j = pos[m - 1 - h];                                                           \
          if (i >= n || j >= n) continue;                                                               \
          if (i > j) { const int t = i; i = j; j = t; }                                                 \
          T *x = W + (size_t)i * n, *y = W + (size_t)j * n;                                             \
          T a = 0, b = 0, c = 0;                                                                        \
          for (int l = 0; l < n; ++l) { a += x[l] * x[l]; b += y[l] * y[l]; c += x[l] * y[l]; }         \
          if (c == 0 || FABS(c) <= tol * SQRT(a * b)) continue;                                         \
          T cs, sn;                                                                                     \
          if (J[i] == J[j]) {                                                                           \
            const T z = (b - a) / (2 * c);                                                              \
            const T t = (z >= 0 ? 1 : -1) / (FABS(z) + SQRT(1 + z * z));                               \
            cs = 1 / SQRT(1 + t * t);                                                                   \
            sn = cs * t;                                                                                \
            for (int l = 0; l < n; ++l) {                                                               \
              const T u = x[l], v = y[l];                                                               \
              x[l] = cs * u - sn * v;                                                                   \
              y[l] = sn * u + cs * v;                                                                   \
            }                                                                                           \
          }                                                                                             \
          else {                                                                                        \
            /* x' = ch x + sh y, y' = sh x + ch y; <x', y'> = 0 at tanh 2t = -2c / (a + b) */           \
            const T z = -(a + b) / (2 * c);                                                             \
            const T t = (z >= 0 ? 1 : -1) / (FABS(z) + SQRT(z * z - 1));                               \
            cs = 1 / SQRT(1 - t * t);                                                                   \
            sn = cs * t;                                                                                \
            for (int l = 0; l < n; ++l) {                                                               \
              const T u = x[l], v = y[l];                                                               \
              x[l] = cs * u + sn * v;                                                                   \
              y[l] = sn * u + cs * v;                                                                   \
            }                                                                                           \
          }                                                                                             \
          rotated += 1;                                                                                 \
        }                                                                                               \
        /* round-robin: keep pos[0], rotate the rest */                                                \
        const int last = pos[m - 1];                                                                    \
        for (int k = m - 1; k > 1; --k) pos[k] = pos[k - 1];                                            \
        pos[1] = last;                                                                                  \
      }                                                                                                 \
      done = (rotated == 0);                                                                            \
    }                                                                                                   \
    for (int j = 0; j < n; ++j) {                                                                       \
      T a = 0;                                                                                          \
      for (int l = 0; l < n; ++l) a += W[(size_t)j * n + l] * W[(size_t)j * n + l];                    \
      sigma[j] = (double)SQRT(a);                                                                       \
    }                                                                                                   \
    free(W);                                                                                            \
    free(pos);                                                                                          \
    return done ? sweep : -1;                                                                           \
  }                                                                                                     \
                                                                                                        \
  /* complex (interleaved re, im): the same iteration on complex columns */                          \
  int jq_zsigma_##SUF(int n, const double *Y, int ldy, const int *J, double *sigma, int nt,            \
                      int max_sweeps)                                                                   \
  {                                                                                                     \
    const int m = n + (n & 1);                                                                          \
    T *W = (T *)malloc(sizeof(T) * 2 * (size_t)n * n);                                                  \
    int *pos = (int *)malloc(sizeof(int) * (size_t)m);                                                  \
    if (!W || !pos) { free(W); free(pos); return -2; }                                                  \
    for (int j = 0; j < n; ++j)                                                                         \
      for (int i = 0; i < 2 * n; ++i) W[(size_t)j * 2 * n + i] = (T)Y[(size_t)j * 2 * ldy + i];         \
    const T tol = (T)n * (T)(U16);                                                                      \
    int sweep = 0, done = 0;                                                                            \
    while (!done && sweep < max_sweeps) {                                                               \
      ++sweep;                                                                                          \
      int rotated = 0;                                                                                  \
      for (int k = 0; k < m; ++k) pos[k] = k;                                                           \
      for (int r = 0; r < m - 1; ++r) {                                                                 \
        _Pragma("omp parallel for num_threads(nt) schedule(dynamic, 1) reduction(+ : rotated)")         \
        for (int h = 0; h < m / 2; ++h) {                                                               \
          int i = pos[h], j = pos[m - 1 - h];                                                           \
          if (i >= n || j >= n) continue;                                                               \
          if (i > j) { const int t = i; i = j; j = t; }                                                 \
          T *x = W + (size_t)i * 2 * n, *y = W + (size_t)j * 2 * n;                                     \
          T a = 0, b = 0, cr = 0, ci = 0; /* c = x^H y */                                               \
          for (int l = 0; l < n; ++l) {                                                                 \
            const T xr = x[2 * l], xi = x[2 * l + 1], yr = y[2 * l], yi = y[2 * l + 1];                 \
            a += xr * xr + xi * xi;                                                                     \
            b += yr * yr + yi * yi;                                                                     \
            cr += xr * yr + xi * yi;                                                                    \
            ci += xr * yi - xi * yr;                                                                    \
          }                                                                                             \
          const T c = SQRT(cr * cr + ci * ci);                                                          \
          if (c == 0 || c <= tol * SQRT(a * b)) continue;                                               \
          /* y := y conj(c) / |c| makes x^H y real and positive */                                     \
          const T er = cr / c, ei = -ci / c;                                                            \
          for (int l = 0; l < n; ++l) {                                                                 \
            const T yr = y[2 * l], yi = y[2 * l + 1];                                                   \
            y[2 * l] = yr * er - yi * ei;                                                               \
            y[2 * l + 1] = yr * ei + yi * er;                                                           \
          }                                                                                             \
          T cs, sn, sgn;                                                                                \
          if (J[i] == J[j]) {                                                                           \
            const T z = (b - a) / (2 * c);                                                              \
            const T t = (z >= 0 ? 1 : -1) / (FABS(z) + SQRT(1 + z * z));                               \
            cs = 1 / SQRT(1 + t * t);                                                                   \
            sn = cs * t;                                                                                \
            sgn = -1;                                                                                   \
          }                                                                                             \
          else {                                                                                        \
            const T z = -(a + b) / (2 * c);                                                             \
            const T t = (z >= 0 ? 1 : -1) / (FABS(z) + SQRT(z * z - 1));                               \
            cs = 1 / SQRT(1 - t * t);                                                                   \
            sn = cs * t;                                                                                \
            sgn = 1;                                                                                    \
          }                                                                                             \
          for (int l = 0; l < 2 * n; ++l) {                                                             \
            const T u = x[l], v = y[l];                                                                 \
            x[l] = cs * u + sgn * sn * v;                                                               \
            y[l] = sn * u + cs * v;                                                                     \
          }                                                                                             \
          rotated += 1;                                                                                 \
        }                                                                                               \
        const int last = pos[m - 1];                                                                    \
        for (int k = m - 1; k > 1; --k) pos[k] = pos[k - 1];                                            \
        pos[1] = last;                                                                                  \
      }                                                                                                 \
      done = (rotated == 0);                                                                            \
    }                                                                                                   \
    for (int j = 0; j < n; ++j) {                                                                       \
      T a = 0;                                                                                          \
      for (int l = 0; l < 2 * n; ++l) a += W[(size_t)j * 2 * n + l] * W[(size_t)j * 2 * n + l];        \
      sigma[j] = (double)SQRT(a);                                                                       \
    }                                                                                                   \
    free(W);                                                                                            \
    free(pos);                                                                                          \
    return done ? sweep : -1;                                                                           \
  }

static long double sqrt_ld(long double x) { return sqrtl(x); }
static long double fabs_ld(long double x) { return fabsl(x); }

JQ_DEFINE(q, __float128, sqrtq, fabsq, 1.6e-33)
JQ_DEFINE(ld, long double, sqrt_ld, fabs_ld, 8.7e-19)
