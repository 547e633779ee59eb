// Test infrastructure for the oracle: an opt-in perturbation of the transcendental functions the
// reference's device code calls (exp, log, pow, log10, sqrt is exact and left alone).
//
// The oracle library is linked with -Bsymbolic-functions, so the reference code's calls to these
// functions bind to the definitions below, which forward to the C library's versions. With the
// perturbation switched on (xref_set_perturbation), every result is moved by one unit in the
// last place, up or down at random. Running a load with and without it measures how strongly
// each output entry depends on the last bit of the elementary functions: two correct
// implementations whose exp/log differ by an ulp (a GPU's and the host C library's, say) can
// legitimately differ by that much, so parity tolerances add a multiple of it.
#include <dlfcn.h>
#include <stdint.h>
#include <string.h>

namespace {

typedef double (*fn1)(double);
typedef double (*fn2)(double, double);
fn1 real_exp = 0, real_log = 0, real_log10 = 0;
fn2 real_pow = 0;
int g_mode = 0;
uint64_t g_state = 0x9e3779b97f4a7c15ULL;

void init() {
  if (real_exp) return;
  void *h = dlopen("libm.so.6", RTLD_NOW | RTLD_LOCAL);
  real_exp = (fn1)dlsym(h, "exp");
  real_log = (fn1)dlsym(h, "log");
  real_log10 = (fn1)dlsym(h, "log10");
  real_pow = (fn2)dlsym(h, "pow");
}

double bump(double v) {
  if (!g_mode) return v;
  uint64_t b;
  memcpy(&b, &v, 8);
  if ((b & 0x7ff0000000000000ULL) == 0x7ff0000000000000ULL || (b << 1) == 0) return v;  // inf, nan, +-0
  g_state = g_state * 6364136223846793005ULL + 1442695040888963407ULL;
  if ((g_state >> 33) & 1)
    b += 1;  // one ulp away from zero
  else
    b -= 1;  // one ulp towards zero
  memcpy(&v, &b, 8);
  return v;
}

}  // namespace

extern "C" {

double exp(double x) {
  init();
  return bump(real_exp(x));
}
double log(double x) {
  init();
  return bump(real_log(x));
}
double log10(double x) {
  init();
  return bump(real_log10(x));
}
double pow(double x, double y) {
  init();
  return bump(real_pow(x, y));
}

// mode 0: exact C-library results; mode 1: each result moved by one ulp, direction from `seed`.
void xref_set_perturbation(int mode, unsigned long long seed) {
  init();
  g_mode = mode;
  g_state = seed * 2654435761ULL + 0x9e3779b97f4a7c15ULL;
}

}  // extern "C"
