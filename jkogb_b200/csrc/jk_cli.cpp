// jk_cli.cpp -- the djk / zjk command-line programs over the C ABI of libjkogb_b200.
//
//   djk FN N N_2 [ID_NCP [ID_TRU]]     (zjk: the complex program, built with -DJK_COMPLEX)
//
// The command line, the files and the messages follow the reference's drivers
// (src/D/djk.F90, src/Z/zjk.F90, src/shared/readcl.F90:1-85, src/shared/binio.F90):
// FN.Y (N x N column-major float64, complex128 for zjk) and FN.J (N int64 signs) are
// read; FN.YU (U), FN.ZZ (Z) and FN.SY (N float64) are written, Y = YU diag(SY) ZZ.
// The step log goes to stderr as DSTEP_LOOP's CSV (src/D/dstep.F90:389-442, 560); the
// steps run on the GPU in CUDA graphs, so its BUILDs column holds the solve's mean time
// per step and TRANSFs 0.  An error ends the program with "STOP <message>" on stderr
// and exit status 1.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/jkogb.h"

namespace {

#ifdef JK_COMPLEX
constexpr int kEl = 2;  // doubles per entry
const char *kProg = "zjk";
#else
constexpr int kEl = 1;
const char *kProg = "djk";
#endif

[[noreturn]] void stop(const std::string &msg)
{
  fprintf(stderr, "STOP %s\n", msg.c_str());
  exit(1);
}

void info_stop(long long info, const char *what)
{
  fprintf(stderr, "INFO=%11lld\n", info);
  stop(what);
}

bool parse_int(const char *s, int &v)
{
  char *e = nullptr;
  const long x = strtol(s, &e, 10);
  if (!e || *e || e == s || x < -2147483647L || x > 2147483647L) return false;
  v = (int)x;
  return true;
}

// JSTEP_LEN, src/shared/jstep.F90:124-133
int jstep_len(int n, int n_2)
{
  if (!n_2) return n / 2;
  const int a = (n_2 > 0) ? n_2 : 0;
  return (a < n / 2) ? a : n / 2;
}

// Fortran ES25.17E3: 17 digits after the point, a three-digit exponent, width 25
std::string es25(double x)
{
  char b[64];
  if (std::isnan(x)) return std::string(22, ' ') + "NaN";
  if (std::isinf(x)) return std::string(x < 0 ? 21 : 22, ' ') + (x < 0 ? "-Inf" : "Inf");
  snprintf(b, sizeof b, "%.17E", x);
  std::string s(b);
  const size_t e = s.find('E');
  const char sign = s[e + 1];
  int ex = atoi(s.c_str() + e + 2);
  char t[16];
  snprintf(t, sizeof t, "E%c%03d", sign, ex);
  s = s.substr(0, e) + t;
  if (s.size() < 25) s = std::string(25 - s.size(), ' ') + s;
  return s;
}

template <typename T>
bool read_file(const std::string &name, std::vector<T> &v, size_t count)
{
  FILE *f = fopen(name.c_str(), "rb");
  if (!f) return false;
  v.resize(count);
  const size_t got = fread(v.data(), sizeof(T), count, f);
  fclose(f);
  return got == count;
}

template <typename T>
bool write_file(const std::string &name, const T *p, size_t count)
{
  FILE *f = fopen(name.c_str(), "wb");
  if (!f) return false;
  const size_t put = fwrite(p, sizeof(T), count, f);
  return (fclose(f) == 0) && put == count;
}

}  // namespace

int main(int argc, char **argv)
{
  // READCL, src/shared/readcl.F90
  int n = 0, n_2 = 0, id_ncp = 0, id_tru = 0;
  if (argc < 4 || argc > 6 || !parse_int(argv[2], n) || !parse_int(argv[3], n_2) ||
      (argc > 4 && !parse_int(argv[4], id_ncp)) || (argc > 5 && !parse_int(argv[5], id_tru)))
    stop(std::string(kProg) + ".exe FN N N_2 [ID_NCP [ID_TRU]]");
  const std::string fn = argv[1];
  if (n <= 2) stop("N should be at least 3 (for N=2 use dtest)");
  n_2 = jstep_len(n, n_2);
  if (n_2 <= 0) stop("JSTEP_LEN");
  if (id_ncp < 0 || id_ncp > 3 || id_tru < 0 || id_tru > 2) stop("DPROC_INIT");

  const size_t nn = (size_t)n * n;
  std::vector<double> A;
  std::vector<long long> J64;
  if (!read_file(fn + ".Y", A, nn * kEl)) info_stop(1, "OPEN_YJ_RO");
  if (!read_file(fn + ".J", J64, (size_t)n)) info_stop(2, "OPEN_YJ_RO");
  std::vector<int> J(n);
  int np = 0, nm = 0;
  for (int i = 0; i < n; ++i) {
    if (J64[i] == 1) ++np;
    else if (J64[i] == -1) ++nm;
    else info_stop(JK_ERR_J, "R%TRU");
    J[i] = (int)J64[i];
  }
  const long long tt = (long long)np * (np - 1) / 2 + (long long)nm * (nm - 1) / 2;
  printf("J has%11d +  and%11d - signs for <=%11lld trig. transfs.\n", np, nm, tt);
  fflush(stdout);

  std::vector<double> U(nn * kEl), Z(nn * kEl), S(n);
  // the step log: capacity for the steps of a typical solve; longer solves log their start
  const int cap = (n < 4096) ? 200 * n + 100000 : 1 << 20;
  std::vector<int> sl(cap), nl(cap), tg(cap), hy(cap);
  std::vector<double> tw(cap);
  jk_trace tr;
  memset(&tr, 0, sizeof tr);
  tr.max_steps = cap;
  tr.sl = sl.data();
  tr.nl = nl.data();
  tr.trig = tg.data();
  tr.hyp = hy.data();
  tr.tw = tw.data();

  const auto t0 = std::chrono::steady_clock::now();
#ifdef JK_COMPLEX
  const int info = jk_zstep_loop(n, U.data(), n, A.data(), n, Z.data(), n, J.data(), S.data(), n_2, id_ncp, id_tru,
                                 nullptr, &tr);
#else
  const int info = jk_dstep_loop(n, U.data(), n, A.data(), n, Z.data(), n, J.data(), S.data(), n_2, id_ncp, id_tru,
                                 nullptr, &tr);
#endif
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

  fprintf(stderr, "\"STEP\",\"OLDLEN\",\"BUILDs\",\"TRANSFs\",\"NEWLEN\",\"NORMF2D\",\"TRIG\",\"HYP\"\n");
  const int rows = (tr.n_steps < cap) ? tr.n_steps : cap;
  const double per = (rows > 0) ? secs / rows : 0.0;
  for (int s = 0; s < rows; ++s) {
    if (sl[s] <= 0)  // the last step: no pivots
      fprintf(stderr, "%11d,%11d,%12.6f,%12.6f,%11d,%s,%11d,%11d\n", s, sl[s], per, 0.0, -1, es25(-0.0).c_str(), 0, 0);
    else
      fprintf(stderr, "%11d,%11d,%12.6f,%12.6f,%11d,%s,%11d,%11d\n", s, sl[s], per, 0.0, nl[s], es25(tw[s]).c_str(), tg[s],
              hy[s]);
  }
  if (tr.n_steps > cap) fprintf(stderr, "(%d further steps not logged)\n", tr.n_steps - cap);
  if (info >= 0) printf("Executed %11d steps with transformations in %13.6f s\n", info, secs);
  else fprintf(stderr, "ERROR %11d after %13.6f s\n", info, secs);
  fflush(stdout);
  fflush(stderr);
  if (info <= JK_ERR_CUDA && info >= JK_ERR_NO_DEVICE) info_stop(info, jk_strerror(info));

  if (!write_file(fn + ".YU", U.data(), nn * kEl)) info_stop(1, "OPEN_UZS_WO");
  if (!write_file(fn + ".ZZ", Z.data(), nn * kEl)) info_stop(2, "OPEN_UZS_WO");
  if (!write_file(fn + ".SY", S.data(), (size_t)n)) info_stop(3, "OPEN_UZS_WO");
  return 0;
}
