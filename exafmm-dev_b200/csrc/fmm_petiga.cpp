// The PetIGA wrapper ABI (wrappers/petiga.cxx:45-316) over the fmm_b200 C ABI, for one rank
// on one GPU.  It is a library of its own (libexafmm_b200_petiga.so, linked against
// libexafmm_b200.so) because its FMM_Init / FMM_Partition / FMM_Finalize share their names
// with the gromacs wrapper's, as the reference's wrappers do.
//
// Two body sets, "b" and "v", are kept from FMM_Init (positions and charges as separate x,
// y, z, value arrays).  Single-rank semantics: FMM_Partition's bisection and body exchange
// are identities (positions come back unchanged, in the same order), and the trees of
// FMM_BuildTree are built by every call from the same positions, which gives the same
// trees.  Each interaction call sets the charges it is given and adds the potential per unit
// target charge to its output array, as the reference does (:141-280):
//   B2B(vi, vb): b on b with charges vb, into vi
//   V2B(vb, vv): v (charges vv) on b, into vb     (two trees, each on its own box)
//   B2V(vv, vb): b (charges vb) on v, into vv     (two trees, each on its own box)
//   V2V(vi, vv): v on v with charges vv, into vi
//   Direct(...): the direct sum of sources j on targets i, into vi (FP64 on the GPU).
// Parameters as the reference's FMM_Init (:45-92): nspawn 1000, theta 0.4, use_rmax and
// use_ropt on, images 0, eps2 stored as an integer (Traversal::eps2 is `const int`), the
// given ncrit; spherical basis at EXAFMM_B200_P (default 10) in FP32.
#include <cstdio>
#include <cstdlib>
#include <vector>

#define EXAFMM_B200_NO_GROMACS_ABI
#include "../../include/exafmm_b200.h"
#include "../../include/exafmm_b200_petiga.h"

namespace {

struct BodySet {
  std::vector<double> x, q;  // x: 3 per body
  void set(int n, const double* xs, const double* ys, const double* zs, const double* v) {
    x.resize(3 * (size_t)n);
    q.assign(v, v + n);
    for (int i = 0; i < n; i++) {
      x[3 * (size_t)i] = xs[i];
      x[3 * (size_t)i + 1] = ys[i];
      x[3 * (size_t)i + 2] = zs[i];
    }
  }
  int n() const { return (int)q.size(); }
};

BodySet g_b, g_v;
fmm_b200_solver* g_solver = nullptr;
double g_eps2 = 0;

int env_order() {
  const char* e = std::getenv("EXAFMM_B200_P");
  return e ? std::atoi(e) : 10;
}

void report(int rc, const char* what) {
  if (rc != FMM_OK)
    std::fprintf(stderr, "exafmm_b200 petiga: %s failed (%d): %s\n", what, rc,
                 fmm_b200_last_error(g_solver));
}

// targets t (charges qt) from sources s (charges qs): potential per unit target charge added
// to out[i]; same = the one-tree solve of a set on itself
void interact(const BodySet& t, const std::vector<double>& qt, const BodySet& s,
              const std::vector<double>& qs, bool same, double* out) {
  if (!g_solver || t.n() == 0) return;
  std::vector<double> p(t.n()), f(3 * (size_t)t.n());
  const int rc = same ? fmm_b200_solve_host(g_solver, t.n(), t.x.data(), qt.data(), p.data(),
                                            f.data())
                      : fmm_b200_solve_ij_host(g_solver, t.n(), t.x.data(), qt.data(), s.n(),
                                               s.x.data(), qs.data(), 0, p.data(), f.data());
  report(rc, "solve");
  if (rc != FMM_OK) return;
  for (int i = 0; i < t.n(); i++) out[i] += p[i];
}

}  // namespace

extern "C" {

void FMM_Init(double eps2, int ncrit, int threads, int nb, double* xb, double* yb, double* zb,
              double* vb, int nv, double* xv, double* yv, double* zv, double* vv) {
  (void)threads;
  if (g_solver) fmm_b200_destroy(g_solver);
  g_solver = nullptr;
  g_eps2 = (double)(int)eps2;
  g_b.set(nb, xb, yb, zb, vb);
  g_v.set(nv, xv, yv, zv, vv);
  fmm_b200_config cfg;
  fmm_b200_default_config(&cfg);
  cfg.P = env_order();
  cfg.theta = 0.4;
  cfg.ncrit = ncrit;
  cfg.nspawn = 1000;
  cfg.use_rmax = 1;
  cfg.use_ropt = 1;
  cfg.eps2 = g_eps2;
  cfg.images = 0;
  const int rc = fmm_b200_create(&cfg, &g_solver);
  if (rc != FMM_OK) {
    std::fprintf(stderr, "exafmm_b200 petiga: create failed (%d): %s\n", rc,
                 fmm_b200_last_error(nullptr));
    g_solver = nullptr;
  }
}

void FMM_Finalize(void) {
  if (g_solver) fmm_b200_destroy(g_solver);
  g_solver = nullptr;
}

void FMM_Partition(int& nb, double* xb, double* yb, double* zb, double* vb, int& nv, double* xv,
                   double* yv, double* zv, double* vv) {
  // one rank: the bodies stay where they are
  auto put = [](const BodySet& s, int& n, double* x, double* y, double* z, double* v) {
    n = s.n();
    for (int i = 0; i < n; i++) {
      x[i] = s.x[3 * (size_t)i];
      y[i] = s.x[3 * (size_t)i + 1];
      z[i] = s.x[3 * (size_t)i + 2];
      v[i] = s.q[i];
    }
  };
  put(g_b, nb, xb, yb, zb, vb);
  put(g_v, nv, xv, yv, zv, vv);
}

void FMM_BuildTree(void) {}  // the trees are built by each interaction call

void FMM_B2B(double* vi, double* vb, bool verbose) {
  (void)verbose;
  std::vector<double> q(vb, vb + g_b.n());
  interact(g_b, q, g_b, q, true, vi);
}

void FMM_V2B(double* vb, double* vv, bool verbose) {
  (void)verbose;
  std::vector<double> one(g_b.n(), 1.0), qs(vv, vv + g_v.n());
  interact(g_b, one, g_v, qs, false, vb);
}

void FMM_B2V(double* vv, double* vb, bool verbose) {
  (void)verbose;
  std::vector<double> one(g_v.n(), 1.0), qs(vb, vb + g_b.n());
  interact(g_v, one, g_b, qs, false, vv);
}

void FMM_V2V(double* vi, double* vv, bool verbose) {
  (void)verbose;
  std::vector<double> q(vv, vv + g_v.n());
  interact(g_v, q, g_v, q, true, vi);
}

void Direct(int ni, double* xi, double* yi, double* zi, double* vi, int nj, double* xj,
            double* yj, double* zj, double* vj) {
  BodySet t, s;
  std::vector<double> one(ni, 1.0);
  t.set(ni, xi, yi, zi, one.data());
  s.set(nj, xj, yj, zj, vj);
  std::vector<double> out(4 * (size_t)ni);
  const int rc = fmm_b200_direct(0, ni, t.x.data(), nj, s.x.data(), s.q.data(), g_eps2,
                                 out.data());
  report(rc, "direct");
  if (rc != FMM_OK) return;
  for (int i = 0; i < ni; i++) vi[i] += out[4 * (size_t)i];
}

}  // extern "C"
