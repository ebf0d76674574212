// Host build of the device translation-operator math (exafmm-dev_b200/csrc/fmm_sph_math.cuh,
// fmm_cart_math.cuh), so tests/test_device_math.py can check the exact device arithmetic
// operator by operator against the oracle on the CPU.  Expansions as ncoef doubles.
#include <vector>

#include "fmm_cart_math.cuh"
#include "fmm_sph_math.cuh"

using namespace fmmb200;

namespace {

template <int P> void sph_m2l(const double* Xi, const double* Xj, const double* Mj, double* Li) {
  constexpr int NT = sph::NT(P);
  double yr[NT], yi[NT], Lr[NT] = {}, Lm[NT] = {};
  sph::Angles<double> a = sph::angles(Xi[0] - Xj[0], Xi[1] - Xj[1], Xi[2] - Xj[2]);
  sph::local<double, P>(a, yr, yi);
  // two output ranges, as the FP32 kernel's passes split them
  sph::m2l_pair<double, P, 0, P / 2>(yr, yi, Mj, Lr, Lm);
  sph::m2l_pair<double, P, P / 2, P>(yr, yi, Mj, Lr, Lm);
  for (int t = 0; t < NT; t++) Li[2 * t] += Lr[t], Li[2 * t + 1] += Lm[t];
}
template <int P> void sph_mult(const double* d, double* y) {
  constexpr int NT = sph::NT(P);
  double yr[NT], yi[NT];
  sph::Angles<double> a = sph::angles(d[0], d[1], d[2]);
  sph::multipole<double, P>(a, a.r, yr, yi);
  for (int t = 0; t < NT; t++) y[2 * t] = yr[t], y[2 * t + 1] = yi[t];
}
template <int P> void split(const double* y, double* yr, double* yi) {
  for (int t = 0; t < sph::NT(P); t++) yr[t] = y[2 * t], yi[t] = y[2 * t + 1];
}
// runtime-index terms (the FP64 kernels) and the unrolled ranges (the FP32 kernels) agree
template <int P> void sph_m2m(const double* Xp, const double* Xc, const double* Mc, double* Mp) {
  double d[3] = {Xp[0] - Xc[0], Xp[1] - Xc[1], Xp[2] - Xc[2]}, y[2 * sph::NT(P)];
  double yr[sph::NT(P)], yi[sph::NT(P)], rng[2 * sph::NT(P)] = {};
  sph_mult<P>(d, y);
  split<P>(y, yr, yi);
  sph::m2m_range<double, P>(yr, yi, Mc, rng);
  for (int j = 0; j < P; j++)
    for (int k = 0; k <= j; k++) {
      double r, i;
      sph::m2m_term<double>(j, k, yr, yi, Mc, r, i);
      const int t = sph::sidx(j, k);
      Mp[2 * t] += (r + rng[2 * t]) / 2;
      Mp[2 * t + 1] += (i + rng[2 * t + 1]) / 2;
      if (r != rng[2 * t] || i != rng[2 * t + 1]) Mp[2 * t] += 1e300;  // must agree exactly
    }
}
template <int P> void sph_l2l(const double* Xc, const double* Xp, const double* Lp, double* Lc) {
  double d[3] = {Xc[0] - Xp[0], Xc[1] - Xp[1], Xc[2] - Xp[2]}, y[2 * sph::NT(P)];
  double yr[sph::NT(P)], yi[sph::NT(P)], rng[2 * sph::NT(P)] = {};
  sph_mult<P>(d, y);
  split<P>(y, yr, yi);
  sph::l2l_range<double, P>(yr, yi, Lp, rng);
  for (int j = 0; j < P; j++)
    for (int k = 0; k <= j; k++) {
      double r, i;
      sph::l2l_term<double>(P, j, k, yr, yi, Lp, r, i);
      const int t = sph::sidx(j, k);
      Lc[2 * t] += (r + rng[2 * t]) / 2;
      Lc[2 * t + 1] += (i + rng[2 * t + 1]) / 2;
      if (r != rng[2 * t] || i != rng[2 * t + 1]) Lc[2 * t] += 1e300;  // must agree exactly
    }
}
template <int P> void sph_p2m(const double* Xc, int nb, const double* xq, double* M) {
  for (int b = 0; b < nb; b++) {
    double d[3] = {xq[4 * b] - Xc[0], xq[4 * b + 1] - Xc[1], xq[4 * b + 2] - Xc[2]};
    double y[2 * sph::NT(P)];
    sph_mult<P>(d, y);
    for (int t = 0; t < sph::NT(P); t++) M[2 * t] += xq[4 * b + 3] * y[2 * t], M[2 * t + 1] -= xq[4 * b + 3] * y[2 * t + 1];
  }
}
template <int P> void sph_l2p(const double* Xc, const double* L, int nb, const double* x, double* trg) {
  for (int b = 0; b < nb; b++)
    sph::l2p_body<double, P>(x[3 * b] - Xc[0], x[3 * b + 1] - Xc[1], x[3 * b + 2] - Xc[2], L,
                             trg[4 * b], trg[4 * b + 1], trg[4 * b + 2], trg[4 * b + 3]);
}

template <int P> void cart_m2l(const double* Xi, const double* Xj, const double* Mj, double* Li) {
  double C[cart::NT(P)];
  double dx = Xi[0] - Xj[0], dy = Xi[1] - Xj[1], dz = Xi[2] - Xj[2];
  double invR2 = 1 / (dx * dx + dy * dy + dz * dz);
  cart::derivs<double, P>(C, dx, dy, dz, invR2, std::sqrt(invR2));
  cart::m2l_pair<double, P>(C, Mj, Li);
}
// runtime-index terms and the unrolled per-child forms (the kernels) agree exactly
template <int P> void cart_m2m(const double* Xp, const double* Xc, const double* Mc, double* Mp) {
  double C[cart::NT(P)], unr[cart::NT(P)] = {};
  C[0] = 1;
  cart::power<double, P>(C, Xp[0] - Xc[0], Xp[1] - Xc[1], Xp[2] - Xc[2]);
  cart::m2m_child<double, P>(C, Mc, unr);
  for (int t = 0; t < cart::NT(P); t++) {
    int nx, ny, nz;
    cart::mi_of(t, nx, ny, nz);
    const double v = cart::m2m_term<double>(nx, ny, nz, C, Mc);
    Mp[t] += v;
    if (v != unr[t]) Mp[t] += 1e300;  // must agree exactly
  }
}
template <int P> void cart_l2l(const double* Xc, const double* Xp, const double* Lp, double* Lc) {
  double C[cart::NT(P)], unr[cart::NT(P)] = {};
  C[0] = 1;
  cart::power<double, P>(C, Xc[0] - Xp[0], Xc[1] - Xp[1], Xc[2] - Xp[2]);
  cart::l2l_child<double, P>(C, Lp, unr);
  for (int t = 0; t < cart::NT(P); t++) {
    int nx, ny, nz;
    cart::mi_of(t, nx, ny, nz);
    const double v = cart::l2l_term<double>(P, nx, ny, nz, C, Lp);
    Lc[t] += v;
    if (v != unr[t]) Lc[t] += 1e300;  // must agree exactly
  }
}
template <int P> void cart_p2m(const double* Xc, int nb, const double* xq, double* M) {
  for (int b = 0; b < nb; b++) {
    double C[cart::NT(P)];
    C[0] = xq[4 * b + 3];
    cart::power<double, P>(C, Xc[0] - xq[4 * b], Xc[1] - xq[4 * b + 1], Xc[2] - xq[4 * b + 2]);
    for (int t = 0; t < cart::NT(P); t++) M[t] += C[t];
  }
}
template <int P> void cart_l2p(const double* Xc, const double* L, int nb, const double* x, double* trg) {
  for (int b = 0; b < nb; b++)
    cart::l2p_body<double, P>(x[3 * b] - Xc[0], x[3 * b + 1] - Xc[1], x[3 * b + 2] - Xc[2], L,
                              trg[4 * b], trg[4 * b + 1], trg[4 * b + 2], trg[4 * b + 3]);
}

}  // namespace

#define SPH_ORDERS(X) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(12)
#define CART_ORDERS(X) X(3) X(4) X(5) X(6) X(7)

extern "C" {
int host_op(int basis, int P, int op, const double* A, const double* B, const double* in,
            int nb, const double* bodies, double* out) {
  // op: 0 m2l(A=Xi, B=Xj, in=Mj), 1 m2m(A=Xp, B=Xc, in=Mc), 2 l2l(A=Xc, B=Xp, in=Lp),
  //     3 p2m(A=Xc, bodies=xq), 4 l2p(A=Xc, in=L, bodies=x)
#define CASE_S(p)                                          \
  if (basis == 0 && P == p) {                              \
    if (op == 0) sph_m2l<p>(A, B, in, out);                \
    else if (op == 1) sph_m2m<p>(A, B, in, out);           \
    else if (op == 2) sph_l2l<p>(A, B, in, out);           \
    else if (op == 3) sph_p2m<p>(A, nb, bodies, out);      \
    else sph_l2p<p>(A, in, nb, bodies, out);               \
    return 0;                                              \
  }
#define CASE_C(p)                                          \
  if (basis == 1 && P == p) {                              \
    if (op == 0) cart_m2l<p>(A, B, in, out);               \
    else if (op == 1) cart_m2m<p>(A, B, in, out);          \
    else if (op == 2) cart_l2l<p>(A, B, in, out);          \
    else if (op == 3) cart_p2m<p>(A, nb, bodies, out);     \
    else cart_l2p<p>(A, in, nb, bodies, out);              \
    return 0;                                              \
  }
  SPH_ORDERS(CASE_S)
  CART_ORDERS(CASE_C)
  return 1;
}
}
