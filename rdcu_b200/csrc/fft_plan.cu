// Host-side FFT planning: radix factorisation and twiddle tables.
#include <cmath>

#include "internal.h"

namespace rdcu {

bool make_line_plan(int L, LinePlan* p) {
  if (L < 1 || L > kMaxLine) return false;
  p->L = L;
  p->nstages = 0;
  int rem = L;
  // larger radices first; the Stockham stage handles any order
  const int radices[] = {8, 4, 2, 3, 5, 7, 11, 13};
  for (int r : radices) {
    while (rem % r == 0) {
      if (p->nstages >= kMaxStages) return false;
      p->radix[p->nstages++] = r;
      rem /= r;
    }
  }
  if (rem != 1) return false;
  int Ns = 1;
  for (int st = 0; st < p->nstages; ++st) {
    p->div_m[st] = make_fastdiv((unsigned)(L / p->radix[st]));
    p->div_ns[st] = make_fastdiv((unsigned)Ns);
    Ns *= p->radix[st];
  }
  return true;
}

void make_twiddles(int L, std::vector<double2>& tw) {
  tw.resize(L);
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int t = 0; t < L; ++t) {
    // reduce the angle to the first octant for accuracy, using exact symmetries
    // of the L-th roots of unity
    long long num = t;  // angle = -2 pi num / L
    long double c, s;
    if (4LL * num == L) {
      c = 0.0L; s = 1.0L;
    } else if (2LL * num == L) {
      c = -1.0L; s = 0.0L;
    } else if (4LL * num == 3LL * L) {
      c = 0.0L; s = -1.0L;
    } else {
      long double ang = two_pi * (long double)num / (long double)L;
      c = cosl(ang);
      s = sinl(ang);
    }
    if (num == 0) { c = 1.0L; s = 0.0L; }
    tw[t] = make_double2((double)c, (double)(-s));
  }
}

}  // namespace rdcu
