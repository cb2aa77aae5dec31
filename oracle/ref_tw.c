/* Test infrastructure: plain-double entry points (for ctypes) to the reference's own
 * trigonometric pair weight in extended precision, src/alt/tweight.c dtw / ztw (a_qp^2 + a_pq^2,
 * complex: the four squared parts summed from the largest down; 0 -> "no transformation"
 * NaN).  Built by ref.mk together with that file, which stays where it lies. */
#include <complex.h>

extern long double dtw(const double Aqp, const double Apq);
extern long double ztw(const double _Complex Aqp, const double _Complex Apq);

double jkref_dtw(double aqp, double apq) { return (double)dtw(aqp, apq); }

double jkref_ztw(double aqp_re, double aqp_im, double apq_re, double apq_im)
{
  return (double)ztw(CMPLX(aqp_re, aqp_im), CMPLX(apq_re, apq_im));
}
