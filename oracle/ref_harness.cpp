// Test infrastructure only: a harness that drives the reference exafmm-dev CPU FMM,
// compiled from the reference's own headers and kernel sources (see oracle/Makefile).
// It is the checker the CPU restatement (oracle/fmm_oracle.c) and the CUDA path are
// compared against, and the "reference" CPU baseline timed by bench.py.  Nothing in the
// product links or calls it.
//
// Pipeline driven exactly as examples/serial.cxx:41-60 drives it:
//   BoundBox::getBounds -> BuildTree::buildTree (adaptive, include/build_tree_tbb.h; with
//   -DREF_UNIFORM the uniform Morton tree of include/build_tree_omp.h, which an OpenMP build
//   without TBB selects, include/build_tree.h:12-13)
//   -> UpDownPass::upwardPass -> Traversal::dualTreeTraversal(cells, cells, cycle, mutual)
//   -> UpDownPass::downwardPass
// with the bodies injected from the caller instead of include/dataset.h.
//
// Interaction lists are recorded by linking ref_record.cpp in place of namespace
// kernel (the reference kernels are compiled with -Dkernel=refkernel and forwarded to).
#include "bound_box.h"
#ifdef REF_UNIFORM
#include "build_tree_omp.h"
#else
#include "build_tree_tbb.h"
#endif
#include "traversal.h"
#include "up_down_pass.h"
#include <omp.h>
#include <cstring>
#include <vector>

namespace refrec {
extern bool enabled;
extern C_iter Ci0, Cj0;
extern long long ncells;
extern double cycle;
extern std::vector<long long> m2l, p2p;
}

struct RefRun {
  Bodies bodies, buffer, jbodies;
  Cells cells, jcells;
  std::vector<int> level;
  std::vector<double> R_built;  // cell radius straight out of buildTree
  double t[8];                  // bounds, tree, upward, traverse, downward, total
  int maxlevel;
};

extern "C" {

int ref_P() { return P; }
int ref_nterm() { return NTERM; }
int ref_fp64() { return sizeof(real_t) == 8; }
int ref_spherical() {
#if Spherical
  return 1;
#else
  return 0;
#endif
}
int ref_mass() {
#if MASS
  return 1;
#else
  return 0;
#endif
}
int ref_uniform() {
#ifdef REF_UNIFORM
  return 1;
#else
  return 0;
#endif
}
int ref_kahan() {
#if KAHAN
  return 1;
#else
  return 0;
#endif
}

// stages: 1 = tree, 2 = +upward, 4 = +traversal, 8 = +downward.
// record: record M2L/P2P lists (forces a serial traversal).
// threads: 0 = serial (no omp parallel region), else omp parallel region with that many threads.
// images, cycle: Traversal's periodic image levels and dualTreeTraversal's cycle.
void* ref_run(int n, const double* x, const double* q, int ncrit, int nspawn, double theta,
              int useRmax, int useRopt, double eps2, int mutual, int stages, int record,
              int threads, int images, double cycle) {
  RefRun* run = new RefRun();
  run->bodies.resize(n);
  for (int i = 0; i < n; i++) {
    Body& B = run->bodies[i];
    B.X[0] = x[3 * i + 0];
    B.X[1] = x[3 * i + 1];
    B.X[2] = x[3 * i + 2];
    B.SRC = q[i];
    B.TRG = 0;
    B.IBODY = i;
    B.IRANK = 0;
    B.ICELL = 0;
    B.WEIGHT = 1;
  }
  run->buffer.reserve(n);
  logger::verbose = false;
  BoundBox boundBox(nspawn);
  BuildTree buildTree(ncrit, nspawn);
  UpDownPass upDownPass(theta, useRmax, useRopt);
  Traversal traversal(nspawn, images, eps2);
  refrec::cycle = cycle;
  refrec::enabled = record != 0;
  refrec::m2l.clear();
  refrec::p2p.clear();
  for (int k = 0; k < 8; k++) run->t[k] = 0;
  if (threads > 0) omp_set_num_threads(threads);
  auto body = [&]() {
    double t0 = omp_get_wtime();
    Bounds bounds = boundBox.getBounds(run->bodies);
    double t1 = omp_get_wtime();
    run->cells = buildTree.buildTree(run->bodies, run->buffer, bounds);
    double t2 = omp_get_wtime();
    run->R_built.resize(run->cells.size());
    for (size_t c = 0; c < run->cells.size(); c++) run->R_built[c] = run->cells[c].R;
    double t3 = t2, t4 = t2, t5 = t2;
    if (stages & 2) {
      upDownPass.upwardPass(run->cells);
      t3 = omp_get_wtime();
    }
    if (stages & 4) {
      refrec::Ci0 = run->cells.begin();
      refrec::Cj0 = run->cells.begin();
      refrec::ncells = run->cells.size();
      traversal.dualTreeTraversal(run->cells, run->cells, cycle, mutual != 0);
      t4 = omp_get_wtime();
    }
    if (stages & 8) {
      upDownPass.downwardPass(run->cells);
      t5 = omp_get_wtime();
    }
    run->t[0] = t1 - t0;
    run->t[1] = t2 - t1;
    run->t[2] = (stages & 2) ? t3 - t2 : 0;
    run->t[3] = (stages & 4) ? t4 - t3 : 0;
    run->t[4] = (stages & 8) ? t5 - t4 : 0;
    run->t[5] = omp_get_wtime() - t0;
  };
  if (threads > 0 && !record) {
#pragma omp parallel
#pragma omp single
    body();
  } else {
    body();
  }
  refrec::enabled = false;
  // cell levels from the parent links (root is cell 0)
  int nc = run->cells.size();
  run->level.assign(nc, 0);
  run->maxlevel = 0;
  for (int c = 0; c < nc; c++) {
    const Cell& C = run->cells[c];
    for (int k = 0; k < C.NCHILD; k++) {
      run->level[C.ICHILD + k] = run->level[c] + 1;
      if (run->level[c] + 1 > run->maxlevel) run->maxlevel = run->level[c] + 1;
    }
  }
  return run;
}

// examples/serial.cxx with IneJ (:30-55): targets and sources in two trees (common_box:
// on the box of their common bounds), both upward passes, dualTreeTraversal(cells, jcells, cycle, false),
// the targets' downward pass (serial; lists recorded).  The getters read the targets.
void* ref_run_ij(int nt, const double* xt, const double* qt, int ns, const double* xs,
                 const double* qs, int ncrit, int nspawn, double theta, int useRmax,
                 int useRopt, double eps2, int common_box) {
  RefRun* run = new RefRun();
  auto fill = [](Bodies& b, int n, const double* x, const double* q) {
    b.resize(n);
    for (int i = 0; i < n; i++) {
      Body& B = b[i];
      B.X[0] = x[3 * i + 0];
      B.X[1] = x[3 * i + 1];
      B.X[2] = x[3 * i + 2];
      B.SRC = q[i];
      B.TRG = 0;
      B.IBODY = i;
      B.IRANK = 0;
      B.ICELL = 0;
      B.WEIGHT = 1;
    }
  };
  fill(run->bodies, nt, xt, qt);
  fill(run->jbodies, ns, xs, qs);
  run->buffer.reserve(nt > ns ? nt : ns);
  logger::verbose = false;
  BoundBox boundBox(nspawn);
  BuildTree buildTree(ncrit, nspawn);
  UpDownPass upDownPass(theta, useRmax, useRopt);
  Traversal traversal(nspawn, 0, eps2);
  for (int k = 0; k < 8; k++) run->t[k] = 0;
  refrec::m2l.clear();
  refrec::p2p.clear();
  // common_box: examples/serial.cxx IneJ; else each tree on its own bounds, as the petiga
  // wrapper builds them (wrappers/petiga.cxx:134-139)
  Bounds bounds = boundBox.getBounds(run->bodies);
  Bounds jbounds = boundBox.getBounds(run->jbodies);
  if (common_box) jbounds = bounds = boundBox.getBounds(run->jbodies, bounds);
  run->cells = buildTree.buildTree(run->bodies, run->buffer, bounds);
  run->R_built.resize(run->cells.size());
  for (size_t c = 0; c < run->cells.size(); c++) run->R_built[c] = run->cells[c].R;
  upDownPass.upwardPass(run->cells);
  run->jcells = buildTree.buildTree(run->jbodies, run->buffer, jbounds);
  upDownPass.upwardPass(run->jcells);
  refrec::enabled = true;
  refrec::Ci0 = run->cells.begin();
  refrec::Cj0 = run->jcells.begin();
  refrec::ncells = run->jcells.size();
  traversal.dualTreeTraversal(run->cells, run->jcells, 2 * M_PI, false);
  refrec::enabled = false;
  upDownPass.downwardPass(run->cells);
  int nc = run->cells.size();
  run->level.assign(nc, 0);
  run->maxlevel = 0;
  for (int c = 0; c < nc; c++) {
    const Cell& C = run->cells[c];
    for (int k = 0; k < C.NCHILD; k++) {
      run->level[C.ICHILD + k] = run->level[c] + 1;
      if (run->level[c] + 1 > run->maxlevel) run->maxlevel = run->level[c] + 1;
    }
  }
  return run;
}

void ref_free(void* h) { delete (RefRun*)h; }
int ref_num_cells(void* h) { return ((RefRun*)h)->cells.size(); }
int ref_maxlevel(void* h) { return ((RefRun*)h)->maxlevel; }
void ref_times(void* h, double* t) { std::memcpy(t, ((RefRun*)h)->t, 6 * sizeof(double)); }

void ref_get_cells(void* h, int* iparent, int* ichild, int* nchild, int* ibody, int* nbody,
                   unsigned long long* icell, int* level, double* X, double* R_built, double* R) {
  RefRun* run = (RefRun*)h;
  for (size_t c = 0; c < run->cells.size(); c++) {
    const Cell& C = run->cells[c];
    iparent[c] = C.IPARENT;
    ichild[c] = C.ICHILD;
    nchild[c] = C.NCHILD;
#ifdef REF_UNIFORM
    ibody[c] = (int)(C.BODY - run->bodies.begin());  // the uniform build sets BODY only
#else
    ibody[c] = C.IBODY;
#endif
    nbody[c] = C.NBODY;
    icell[c] = C.ICELL;
    level[c] = run->level[c];
    for (int d = 0; d < 3; d++) X[3 * c + d] = C.X[d];
    R_built[c] = run->R_built[c];
    R[c] = C.R;
  }
}

// Body order after buildTree: original index (IBODY) of each sorted body.
void ref_get_order(void* h, int* ibody) {
  RefRun* run = (RefRun*)h;
  for (size_t b = 0; b < run->bodies.size(); b++) ibody[b] = run->bodies[b].IBODY;
}

// Expansions: which = 0 -> M, 1 -> L.  Spherical: NTERM complex (re, im) pairs per cell;
// Cartesian: NTERM reals per cell.
void ref_get_expansion(void* h, int which, double* out) {
  RefRun* run = (RefRun*)h;
  size_t k = 0;
  for (size_t c = 0; c < run->cells.size(); c++) {
    const Cell& C = run->cells[c];
    for (int i = 0; i < NTERM; i++) {
#if Spherical
      complex_t v = which == 0 ? C.M[i] : C.L[i];
      out[k++] = std::real(v);
      out[k++] = std::imag(v);
#else
      out[k++] = which == 0 ? C.M[i] : C.L[i];
#endif
    }
  }
}

// Potential and gradient per ORIGINAL body index, as the reference leaves them after the
// downward pass (per unit target charge: kernel::L2P divides by SRC).
void ref_get_trg(void* h, double* trg) {
  RefRun* run = (RefRun*)h;
  for (size_t b = 0; b < run->bodies.size(); b++) {
    const Body& B = run->bodies[b];
    for (int d = 0; d < 4; d++) trg[4 * B.IBODY + d] = (double)(real_t)B.TRG[d];
  }
}

long long ref_num_m2l() { return refrec::m2l.size(); }
long long ref_num_p2p() { return refrec::p2p.size(); }
// pairs packed as (target << 32) | source | image << 27 (image code of the shift, 0 for
// none), in the order the reference visited them; the M2L of traversePeriodic from cells
// outside the tree are not recorded
void ref_get_m2l(long long* out) { std::memcpy(out, refrec::m2l.data(), refrec::m2l.size() * 8); }
void ref_get_p2p(long long* out) { std::memcpy(out, refrec::p2p.data(), refrec::p2p.size() * 8); }

// The translation-operator chain of examples/kernel.cxx:5-93 (with the eps2 argument the
// stale P2P call at kernel.cxx:77 lacks), returning the rel-L2 potential error of
// P2M -> M2M -> M2L -> L2L -> L2P against P2P.  seed < 0 restores glibc's unseeded
// drand48 state (X = 0), which is what a fresh kernel.cxx process draws from.
double ref_kernel_chain(long seed) {
  if (seed >= 0) {
    srand48(seed);
  } else {
    unsigned short x0[3] = {0, 0, 0};
    seed48(x0);
  }
  Bodies bodies(16), bodies2(16), jbodies(16);
  Cells cells(4);
  vec3 Xperiodic = 0;
  const real_t theta = 0.5;
  const real_t R = 2 / theta;
  for (B_iter B = jbodies.begin(); B != jbodies.end(); B++) {
    B->X[0] = 2 * drand48();
    B->X[1] = 2 * drand48();
    B->X[2] = 2 * drand48();
    B->SRC = drand48();
  }
  C_iter Cj = cells.begin();
  Cj->X = 1;
  Cj->BODY = jbodies.begin();
  Cj->NBODY = jbodies.size();
  Cj->M = 0;
  refrec::enabled = false;
  kernel::P2M(Cj);
  C_iter CJ = cells.begin() + 1;
  CJ->ICHILD = Cj - cells.begin();
  CJ->NCHILD = 1;
  CJ->X = 0;
  CJ->M = 0;
  kernel::M2M(CJ, cells.begin());
  C_iter CI = cells.begin() + 2;
  CI->X = R + 4;
  CI->M = 1;
  CI->L = 0;
#if MASS
  for (int i = 1; i < NTERM; i++) CJ->M[i] /= CJ->M[0];
#endif
  kernel::M2L(CI, CJ, Xperiodic, false);
  C_iter Ci = cells.begin() + 3;
  Ci->X = R + 3;
  Ci->IPARENT = 2;
  Ci->M = 1;
  Ci->L = 0;
  kernel::L2L(Ci, cells.begin());
  for (B_iter B = bodies.begin(); B != bodies.end(); B++) {
    B->X[0] = R + 2 + 2 * drand48();
    B->X[1] = R + 2 + 2 * drand48();
    B->X[2] = R + 2 + 2 * drand48();
    B->SRC = drand48();
    B->TRG = 0;
  }
  Ci->BODY = bodies.begin();
  Ci->NBODY = bodies.size();
  kernel::L2P(Ci);
  for (B_iter B = bodies2.begin(); B != bodies2.end(); B++) {
    *B = bodies[B - bodies2.begin()];
    B->TRG = 0;
  }
  Cj->NBODY = jbodies.size();
  Ci->NBODY = bodies2.size();
  Ci->BODY = bodies2.begin();
  kernel::P2P(Ci, Cj, 0, Xperiodic, false);
  for (B_iter B = bodies2.begin(); B != bodies2.end(); B++) B->TRG /= B->SRC;
  double diff = 0, norm = 0;
  for (B_iter B = bodies.begin(), B2 = bodies2.begin(); B != bodies.end(); B++, B2++) {
    diff += (B->TRG[0] - B2->TRG[0]) * (B->TRG[0] - B2->TRG[0]);
    norm += B2->TRG[0] * B2->TRG[0];
  }
  return std::sqrt(diff / norm);
}

// Single-operator access for kernel-level parity (one cell pair per call).
// cellbuf layout per cell: X[3], R, M (NTERM complex or real), L (same).
}
