// Per-class arithmetic of one primitive quartet of the float32 ERI kernels, counted on the host
// by running the kernels' own shell-quartet code (eri_sq.cuh, B2Sq<T,...>::quartet with its Boys
// evaluation) on a counting number type.  Writes eri_flops.h, which bench.py's ERI roofline uses:
//
//   nvcc -std=c++17 -I. -I../../include -x cu eri_flops_count.cu -o /tmp/eri_flops && /tmp/eri_flops > eri_flops.h
//
// Counting rules: +, -, * and / count one flop each (a fused multiply-add is two); sqrt, exp and
// the reciprocal square root count one each (special-function unit); operations whose operands
// are compile-time constants of the template (the zeros and ones the class's angular momenta fix)
// are folded, as the compiler folds them, and not counted; comparisons and index arithmetic are
// not counted.  The Boys function is counted on its table branch (T < 40), the common one, and
// F_0 alone on its error-function branch (erf counts as one special function).
#include <cstdio>
#include <cmath>
#include "eri_sq.cuh"

static long long g_flops = 0, g_special = 0;

struct CF {                   // value (for the branches) + "is a folded constant" flag
  double v = 0;
  bool k = false;
  CF() = default;
  CF(int x) : v(x), k(true) {}
  CF(double x) : v(x), k(true) {}
  CF(float x) : v(x), k(true) {}
  static CF var(double x) { CF c; c.v = x; c.k = false; return c; }
  explicit operator int() const { return (int)v; }
};
static CF op(double v, bool both_const) {
  CF c;
  c.v = v;
  c.k = both_const;
  if (!both_const) ++g_flops;
  return c;
}
inline CF operator+(CF a, CF b) {
  if (a.k && a.v == 0) return b;
  if (b.k && b.v == 0) return a;
  return op(a.v + b.v, a.k && b.k);
}
inline CF operator-(CF a, CF b) {
  if (b.k && b.v == 0) return a;
  return op(a.v - b.v, a.k && b.k);
}
inline CF operator-(CF a) { CF c = a; c.v = -a.v; return c; }     // sign flips fold into the next op
inline CF operator*(CF a, CF b) {
  if ((a.k && a.v == 0) || (b.k && b.v == 0)) return CF(0);
  if (a.k && a.v == 1) return b;
  if (b.k && b.v == 1) return a;
  return op(a.v * b.v, a.k && b.k);
}
inline CF operator/(CF a, CF b) { return op(a.v / b.v, a.k && b.k); }
inline CF &operator+=(CF &a, CF b) { a = a + b; return a; }
inline CF &operator-=(CF &a, CF b) { a = a - b; return a; }
inline CF &operator*=(CF &a, CF b) { a = a * b; return a; }
inline bool operator<(CF a, CF b) { return a.v < b.v; }
inline bool operator>(CF a, CF b) { return a.v > b.v; }
inline bool operator==(CF a, CF b) { return a.v == b.v; }
inline bool operator!=(CF a, CF b) { return a.v != b.v; }
inline CF sqrt(CF a) { if (!a.k) ++g_special; CF c = a; c.v = std::sqrt(a.v); return c; }
inline CF exp(CF a) { if (!a.k) ++g_special; CF c = a; c.v = std::exp(a.v); return c; }
inline CF erf(CF a) { if (!a.k) ++g_special; CF c = a; c.v = std::erf(a.v); return c; }

// the float32 kernels' Taylor length of the Boys table branch, and their error-function F_0
template <> struct B2BoysTerms<CF> { static constexpr int n = B2BoysTerms<float>::n; };
template <> struct B2BoysErfF0<CF> { static constexpr bool value = B2BoysErfF0<float>::value; };

template <int LI, int LJ, int LK, int LL>
static void count(long long &fl, long long &sp) {
  using S = B2Sq<CF, LI, LJ, LK, LL, -1>;
  static CF tab[B2_BOYS_NT * B2_BOYS_NM];
  static bool filled = false;
  if (!filled) {
    static double t64[B2_BOYS_NT * B2_BOYS_NM];
    b2_boys_fill_table(t64);
    for (int i = 0; i < B2_BOYS_NT * B2_BOYS_NM; ++i) tab[i] = CF::var(t64[i]);
    filled = true;
  }
  B2PairPrim<CF> A, B;
  const double a[12] = {1.3, 0.4, 0.2, -0.1, 0.3, 0.25, -0.2, 0.1, 0.9, 0.35, 0.7, 0.6};
  CF *pa = &A.zeta, *pb = &B.zeta;             // the struct is a run of T fields
  for (int i = 0; i < (int)(sizeof(A) / sizeof(CF)); ++i) {
    pa[i] = CF::var(a[i % 12] + 0.01 * i);
    pb[i] = CF::var(a[(i + 5) % 12] - 0.02 * i);
  }
  CF acc[S::NI][S::NJ][S::NK][S::NL];
  S::zero(acc);
  for (int x = 0; x < S::NI; ++x)
    for (int y = 0; y < S::NJ; ++y)
      for (int z = 0; z < S::NK; ++z)
        for (int w = 0; w < S::NL; ++w) acc[x][y][z][w] = CF::var(0.0);
  g_flops = g_special = 0;
  S::quartet(A, B, tab, acc);
  fl = g_flops;
  sp = g_special;
}

int main() {
  long long f[16], s[16];
#define C(g, LI, LJ, LK, LL) count<LI, LJ, LK, LL>(f[g], s[g]);
  C(0, 0, 0, 0, 0) C(1, 0, 0, 1, 0) C(2, 0, 0, 0, 1) C(3, 0, 0, 1, 1)
  C(4, 1, 0, 0, 0) C(5, 1, 0, 1, 0) C(6, 1, 0, 0, 1) C(7, 1, 0, 1, 1)
  C(8, 0, 1, 0, 0) C(9, 0, 1, 1, 0) C(10, 0, 1, 0, 1) C(11, 0, 1, 1, 1)
  C(12, 1, 1, 0, 0) C(13, 1, 1, 1, 0) C(14, 1, 1, 0, 1) C(15, 1, 1, 1, 1)
#undef C
  printf("// Generated by eri_flops_count.cu from eri_sq.cuh: arithmetic of one primitive quartet of the\n");
  printf("// float32 ERI kernels per class combination g = (lI + 2 lJ) * 4 + (lK + 2 lL) (flops: +, -, *, /;\n");
  printf("// special: sqrt, exp, reciprocal square root), constants folded as the compiler folds them.\n");
  printf("#pragma once\n");
  printf("static const int B2_ERI_FLOPS[16] = {");
  for (int g = 0; g < 16; ++g) printf("%lld%s", f[g], g < 15 ? ", " : "};\n");
  printf("static const int B2_ERI_SPECIAL[16] = {");
  for (int g = 0; g < 16; ++g) printf("%lld%s", s[g], g < 15 ? ", " : "};\n");
  return 0;
}
