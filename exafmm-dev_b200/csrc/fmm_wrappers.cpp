// The reference's wrapper ABI as shims over the fmm_b200 C ABI, for one rank on one GPU.
//
// gromacs (wrappers/gromacs.cxx:28-162): FMM_Init / FMM_Partition / FMM_Coulomb /
// FMM_Finalize with process-global state, as the reference keeps it (:15-26).
// CHARMM (wrappers/charmm.cxx:31-202): fmm_init_ / fmm_partition_ / fmm_coulomb_ /
// fmm_finalize_, Fortran by-reference arguments, icpumap marking local bodies.
//
// Single-rank semantics: the MPI partition and LET exchange are identities, so
// FMM_Partition / fmm_partition_ leave positions and ownership as they are (the reference
// wraps, partitions and unwraps them).  FMM_Coulomb keeps the reference's arithmetic
// around the solve: positions wrapped into [-cycle/2, cycle/2] (vec.h wrap, :193-204),
// incoming p and f taken as initial TRG values (which kernel::L2P then divides by the
// charge), the dipole correction of UpDownPass::dipoleCorrection (up_down_pass.h:160-168)
// applied with the given cycle, and p / f overwritten per original index.  Periodic
// images (FMM_Init's images > 0) are the solver's own: the 27 nearest copies through the
// tree and images - 1 levels of super-cells through the root multipole.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../../include/exafmm_b200.h"

namespace {

fmm_b200_solver* g_solver = nullptr;
bool g_verbose = false;
int g_images = 0;  // periodic image levels given to FMM_Init / fmm_init_

int env_order() {
  const char* e = std::getenv("EXAFMM_B200_P");
  return e ? std::atoi(e) : 10;
}

void init_solver(int images, double theta, int ncrit, bool verbose) {
  if (g_solver) {
    fmm_b200_destroy(g_solver);
    g_solver = nullptr;
  }
  g_verbose = verbose;
  g_images = images;
  fmm_b200_config cfg;
  fmm_b200_default_config(&cfg);
  cfg.P = env_order();
  cfg.theta = theta;
  cfg.ncrit = ncrit;
  cfg.nspawn = 1000;
  cfg.use_rmax = 1;
  cfg.use_ropt = 1;
  cfg.eps2 = 0.0;
  cfg.images = images;
  int rc = fmm_b200_create(&cfg, &g_solver);
  if (rc != FMM_OK) {
    std::fprintf(stderr, "exafmm_b200: create failed (%d): %s\n", rc, fmm_b200_last_error(nullptr));
    g_solver = nullptr;
  }
}

double wrap1(double v, double w) {
  if (v < -w / 2) v += w;
  if (v > w / 2) v -= w;
  return v;
}

// solve bodies (x: 3n wrapped positions, q: n) -> phi, grad phi per body (trg: 4n), with
// the periodic images of the box of side cycle when images > 0
bool solve(int n, const std::vector<double>& x, const std::vector<double>& q, double cycle,
           std::vector<double>& trg) {
  if (!g_solver) return false;
  trg.assign(4 * (size_t)n, 0.0);
  std::vector<double> p(n), f(3 * (size_t)n);
  int rc = fmm_b200_set_periodic(g_solver, g_images, cycle);
  if (rc == FMM_OK) rc = fmm_b200_solve_host(g_solver, n, x.data(), q.data(), p.data(), f.data());
  if (rc != FMM_OK) {
    std::fprintf(stderr, "exafmm_b200: solve failed (%d): %s\n", rc, fmm_b200_last_error(g_solver));
    return false;
  }
  for (int i = 0; i < n; i++) {
    trg[4 * i] = p[i];
    for (int d = 0; d < 3; d++) trg[4 * i + 1 + d] = f[3 * i + d];
  }
  return true;
}

}  // namespace

extern "C" {

void FMM_Init(int images) { init_solver(images, 0.4, 32, true); }

void FMM_Finalize(void) {
  if (g_solver) fmm_b200_destroy(g_solver);
  g_solver = nullptr;
}

void FMM_Partition(int& n, int* index, double* x, double* q, double cycle) {
  (void)n;
  (void)index;
  (void)x;
  (void)q;
  (void)cycle;
}

void FMM_Coulomb(int n, double* x, double* q, double* p, double* f, double cycle) {
  if (!g_solver || n <= 0) return;
  std::vector<double> xw(3 * (size_t)n), qv(q, q + n), trg;
  for (int i = 0; i < 3 * n; i++) xw[i] = wrap1(x[i], cycle);
  if (!solve(n, xw, qv, cycle, trg)) return;
  double dip[3] = {0, 0, 0};
  for (int i = 0; i < n; i++)
    for (int d = 0; d < 3; d++) dip[d] += xw[3 * i + d] * q[i];
  const double coef = 4 * M_PI / (3 * cycle * cycle * cycle);
  const double dn = dip[0] * dip[0] + dip[1] * dip[1] + dip[2] * dip[2];
  for (int i = 0; i < n; i++) {
    p[i] = p[i] / q[i] + trg[4 * i] - coef * dn / n / q[i];
    for (int d = 0; d < 3; d++) f[3 * i + d] = f[3 * i + d] / q[i] + trg[4 * i + 1 + d] - coef * dip[d];
  }
}

void fmm_init_(int* images, double* theta, int* verbose) {
  init_solver(*images, *theta, 32, *verbose != 0);
}

void fmm_finalize_(void) { FMM_Finalize(); }

void fmm_partition_(int* nglobal, int* icpumap, double* x, double* q, double* xold,
                    double* cycle) {
  (void)x;
  (void)q;
  (void)xold;
  (void)cycle;
  for (int i = 0; i < *nglobal; i++) icpumap[i] = icpumap[i] == 1 ? 1 : 0;
}

void fmm_coulomb_(int* nglobal, int* icpumap, double* x, double* q, double* p, double* f,
                  double* cycle) {
  const double Celec = 332.0716;
  std::vector<int> local;
  for (int i = 0; i < *nglobal; i++) {
    if (icpumap[i] == 1) local.push_back(i);
    else icpumap[i] = 0;
  }
  const int n = (int)local.size();
  if (!g_solver || n == 0) return;
  std::vector<double> xw(3 * (size_t)n), qv(n), trg;
  for (int k = 0; k < n; k++) {
    int i = local[k];
    for (int d = 0; d < 3; d++) xw[3 * k + d] = wrap1(x[3 * i + d], *cycle);
    qv[k] = q[i];
  }
  if (!solve(n, xw, qv, *cycle, trg)) return;
  double dip[3] = {0, 0, 0};
  for (int k = 0; k < n; k++)
    for (int d = 0; d < 3; d++) dip[d] += xw[3 * k + d] * qv[k];
  const double coef = 4 * M_PI / (3 * *cycle * *cycle * *cycle);
  const double dn = dip[0] * dip[0] + dip[1] * dip[1] + dip[2] * dip[2];
  for (int k = 0; k < n; k++) {
    int i = local[k];
    double t0 = trg[4 * k] - coef * dn / n / qv[k];
    p[i] += t0 * qv[k] * Celec;
    for (int d = 0; d < 3; d++) f[3 * i + d] += (trg[4 * k + 1 + d] - coef * dip[d]) * qv[k] * Celec;
  }
}

}  // extern "C"
