// exafmm_b200.hpp -- C++ facade with the reference's single-node class API, backed by the
// GPU solver of libexafmm_b200.so (C ABI in exafmm_b200.h).
//
// The reference drives one solve as (examples/serial.cxx:46-60)
//     bounds = boundBox.getBounds(bodies);
//     cells  = buildTree.buildTree(bodies, buffer, bounds);
//     upDownPass.upwardPass(cells);
//     traversal.dualTreeTraversal(cells, cells, cycle, mutual);
//     upDownPass.downwardPass(cells);
// and the same calls compile against this header.  The work runs on the device; Bodies
// and Cells are host mirrors, refreshed after each stage:
//   * buildTree permutes `bodies` into tree order in place, as the reference does
//     (include/build_tree_tbb.h:365-374), and returns the cells in the reference layout;
//   * upwardPass refreshes each Cell's R and M; downwardPass its L and every Body's TRG
//     (phi, grad phi per unit charge, include/types.h:71 and kernels/*CPU.cxx L2P).
// Run-time parameters replace the reference's compile-time ones (EXPANSION, Spherical /
// Cartesian, FP64, include/types.h:12-45): set them in a Context before building.
// Periodic images (spherical basis) and mutual traversals are supported (mutual: the
// reference's set of unordered cell pairs, each evaluated in both directions from the
// target side on the device).  Traversal::direct runs the FP64 direct sum on the GPU (one
// call per periodic shift).
#pragma once
#include <algorithm>
#include <complex>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "exafmm_b200.h"

namespace exafmm_b200 {

typedef double real_t;
typedef std::complex<double> complex_t;

struct vec3 {
  real_t v[3] = {0, 0, 0};
  real_t& operator[](int i) { return v[i]; }
  const real_t& operator[](int i) const { return v[i]; }
};
struct vec4 {
  real_t v[4] = {0, 0, 0, 0};
  real_t& operator[](int i) { return v[i]; }
  const real_t& operator[](int i) const { return v[i]; }
};

struct Bounds {  // include/types.h:54-57
  vec3 Xmin, Xmax;
};

struct Body {  // include/types.h:60-72
  vec3 X;
  real_t SRC = 0;
  int IBODY = 0;
  int IRANK = 0;
  uint64_t ICELL = 0;
  real_t WEIGHT = 1;
  vec4 TRG;
};
typedef std::vector<Body> Bodies;
typedef Bodies::iterator B_iter;

struct Cell {  // include/types.h:79-92 (BODY is an index-based iterator here)
  int IPARENT = 0, ICHILD = 0, NCHILD = 0, IBODY = 0, NBODY = 0;
  B_iter BODY;
  uint64_t ICELL = 0;
  real_t WEIGHT = 0;
  vec3 X;
  real_t R = 0;
  std::vector<complex_t> M, L;  // spherical: NTERM complex; Cartesian: NTERM real parts
};
typedef std::vector<Cell> Cells;
typedef Cells::iterator C_iter;

class Error : public std::runtime_error {
 public:
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Solver parameters the reference fixes at compile time, plus the device.
struct Context {
  fmm_b200_config cfg;
  std::shared_ptr<fmm_b200_solver> solver;
  std::shared_ptr<fmm_b200_solver> ksolver;  // the handle of the namespace kernel calls
  Bodies* bodies = nullptr;
  Context() { fmm_b200_default_config(&cfg); }
  static Context& global() {
    static Context c;
    return c;
  }
  void check(int rc) const {
    if (rc != FMM_OK)
      throw Error(rc, fmm_b200_last_error(solver ? solver.get() : nullptr));
  }
  fmm_b200_solver* get() {
    if (!solver) {
      fmm_b200_solver* s = nullptr;
      int rc = fmm_b200_create(&cfg, &s);
      if (rc != FMM_OK) throw Error(rc, fmm_b200_last_error(nullptr));
      solver.reset(s, [](fmm_b200_solver* p) { fmm_b200_destroy(p); });
    }
    return solver.get();
  }
  void reset() { solver.reset(); }
  fmm_b200_solver* kget() {
    if (!ksolver) {
      fmm_b200_solver* s = nullptr;
      int rc = fmm_b200_create(&cfg, &s);
      if (rc != FMM_OK) throw Error(rc, fmm_b200_last_error(nullptr));
      ksolver.reset(s, [](fmm_b200_solver* p) { fmm_b200_destroy(p); });
    }
    return ksolver.get();
  }
};

inline int nterm(const fmm_b200_config& c) {
  return c.basis == FMM_SPHERICAL ? c.P * (c.P + 1) / 2 : c.P * (c.P + 1) * (c.P + 2) / 6;
}

// BoundBox (include/bound_box.h:73-121)
class BoundBox {
 public:
  explicit BoundBox(int nspawn = 1000) : nspawn_(nspawn) {}
  Bounds getBounds(Bodies& bodies) {
    Bounds b;
    if (bodies.empty()) return b;
    b.Xmin = b.Xmax = bodies.front().X;
    return getBounds(bodies, b);
  }
  Bounds getBounds(const Bodies& bodies, Bounds b) {
    for (const Body& B : bodies)
      for (int d = 0; d < 3; d++) {
        b.Xmin[d] = B.X[d] < b.Xmin[d] ? B.X[d] : b.Xmin[d];
        b.Xmax[d] = B.X[d] > b.Xmax[d] ? B.X[d] : b.Xmax[d];
      }
    return b;
  }

 private:
  int nspawn_;
};

// BuildTree (include/build_tree_tbb.h:362-387).  The tree is built from the bodies'
// own bounds on the device (the bounds argument is accepted for API compatibility).
class BuildTree {
 public:
  BuildTree(int ncrit, int nspawn, Context& ctx = Context::global()) : ctx_(ctx) {
    ctx_.cfg.ncrit = ncrit;
    ctx_.cfg.nspawn = nspawn;
  }
  Cells buildTree(Bodies& bodies, Bodies& buffer, Bounds) {
    ctx_.reset();  // parameters may have changed
    fmm_b200_solver* s = ctx_.get();
    const int n = (int)bodies.size();
    std::vector<double> x(3 * (size_t)n), q(n);
    for (int i = 0; i < n; i++) {
      for (int d = 0; d < 3; d++) x[3 * i + d] = bodies[i].X[d];
      q[i] = bodies[i].SRC;
    }
    ctx_.check(fmm_b200_set_bodies_host(s, n, x.data(), q.data()));
    ctx_.check(fmm_b200_build_tree(s));
    std::vector<int> order(n);
    if (n) ctx_.check(fmm_b200_get_order(s, order.data()));
    buffer = bodies;
    for (int i = 0; i < n; i++) bodies[i] = buffer[order[i]];
    ctx_.bodies = &bodies;
    maxlevel_ = 0;
    return fetch_cells(ctx_, bodies, false, false);
  }
  void printTreeData(Cells& cells) { (void)cells; }

  static Cells fetch_cells(Context& ctx, Bodies& bodies, bool M, bool L) {
    fmm_b200_solver* s = ctx.get();
    int nc = 0, ml = 0;
    ctx.check(fmm_b200_num_cells(s, &nc, &ml));
    std::vector<int> ip(nc), ic(nc), nch(nc), ib(nc), nb(nc), lev(nc);
    std::vector<unsigned long long> key(nc);
    std::vector<double> X(3 * (size_t)nc), R(nc);
    if (nc)
      ctx.check(fmm_b200_get_cells(s, ip.data(), ic.data(), nch.data(), ib.data(), nb.data(),
                                   key.data(), lev.data(), X.data(), R.data()));
    const int nt = nterm(ctx.cfg);
    const int w = ctx.cfg.basis == FMM_SPHERICAL ? 2 : 1;
    std::vector<double> em, el;
    if (M && nc) {
      em.resize((size_t)nc * nt * w);
      ctx.check(fmm_b200_get_expansion(s, 0, em.data()));
    }
    if (L && nc) {
      el.resize((size_t)nc * nt * w);
      ctx.check(fmm_b200_get_expansion(s, 1, el.data()));
    }
    Cells cells(nc);
    for (int c = 0; c < nc; c++) {
      Cell& C = cells[c];
      C.IPARENT = ip[c];
      C.ICHILD = ic[c];
      C.NCHILD = nch[c];
      C.IBODY = ib[c];
      C.NBODY = nb[c];
      C.BODY = bodies.begin() + ib[c];
      C.ICELL = key[c];
      for (int d = 0; d < 3; d++) C.X[d] = X[3 * c + d];
      C.R = R[c];
      auto unpack = [&](const std::vector<double>& e, std::vector<complex_t>& out) {
        if (e.empty()) return;
        out.resize(nt);
        for (int t = 0; t < nt; t++)
          out[t] = w == 2 ? complex_t(e[((size_t)c * nt + t) * 2], e[((size_t)c * nt + t) * 2 + 1])
                          : complex_t(e[(size_t)c * nt + t], 0);
      };
      unpack(em, C.M);
      unpack(el, C.L);
    }
    return cells;
  }

 private:
  Context& ctx_;
  int maxlevel_ = 0;
};

// UpDownPass (include/up_down_pass.h:113-148)
class UpDownPass {
 public:
  UpDownPass(real_t theta, bool useRmax, bool useRopt, Context& ctx = Context::global())
      : ctx_(ctx) {
    ctx_.cfg.theta = theta;
    ctx_.cfg.use_rmax = useRmax;
    ctx_.cfg.use_ropt = useRopt;
  }
  void upwardPass(Cells& cells) {
    if (cells.empty()) return;
    ctx_.check(fmm_b200_upward_pass(ctx_.get()));
    cells = BuildTree::fetch_cells(ctx_, *ctx_.bodies, true, false);
  }
  void downwardPass(Cells& cells) {
    if (cells.empty()) return;
    fmm_b200_solver* s = ctx_.get();
    ctx_.check(fmm_b200_downward_pass(s));
    Bodies& bodies = *ctx_.bodies;
    const int n = (int)bodies.size();
    std::vector<double> trg(4 * (size_t)n);
    std::vector<int> order(n);
    if (n) {
      ctx_.check(fmm_b200_get_trg_host(s, trg.data()));  // caller (pre-sort) order
      ctx_.check(fmm_b200_get_order(s, order.data()));
    }
    for (int b = 0; b < n; b++)
      for (int d = 0; d < 4; d++) bodies[b].TRG[d] = trg[4 * (size_t)order[b] + d];
    cells = BuildTree::fetch_cells(ctx_, bodies, true, true);
  }

 private:
  Context& ctx_;
};

// Traversal (include/traversal.h:214-337).
class Traversal {
 public:
  Traversal(int nspawn, int images, real_t eps2, Context& ctx = Context::global()) : ctx_(ctx) {
    ctx_.cfg.nspawn = nspawn;
    ctx_.cfg.images = images;
    ctx_.cfg.eps2 = (double)(int)eps2;  // the reference stores eps2 as const int (:17)
  }
  void dualTreeTraversal(Cells& icells, Cells& jcells, real_t cycle, bool mutual,
                         real_t remote = 1) {
    (void)jcells;
    (void)remote;
    if (icells.empty()) return;
    ctx_.check(fmm_b200_set_periodic(ctx_.get(), ctx_.cfg.images, (double)cycle));
    ctx_.check(fmm_b200_set_mutual(ctx_.get(), mutual ? 1 : 0));
    ctx_.check(fmm_b200_traverse(ctx_.get()));
  }
  // direct sum on the GPU in FP64: TRG of ibodies += contributions of jbodies
  // (times the target's own charge, as kernel::P2P leaves it before normalize)
  // with periodic images: the shifts (ix, iy, iz) cycle, |i| <= sum_{l < images} 3^l, of
  // the reference's DirectRecursion (:266-301)
  void direct(Bodies& ibodies, Bodies& jbodies, real_t cycle) {
    const int nt = (int)ibodies.size(), ns = (int)jbodies.size();
    std::vector<double> x0(3 * (size_t)nt), xt(3 * (size_t)nt), xs(3 * (size_t)ns), qs(ns),
        out(4 * (size_t)nt), acc(4 * (size_t)nt, 0.0);
    for (int i = 0; i < nt; i++)
      for (int d = 0; d < 3; d++) x0[3 * i + d] = ibodies[i].X[d];
    for (int j = 0; j < ns; j++) {
      for (int d = 0; d < 3; d++) xs[3 * j + d] = jbodies[j].X[d];
      qs[j] = jbodies[j].SRC;
    }
    int prange = 0;
    for (int l = 0, p3 = 1; l < ctx_.cfg.images; l++, p3 *= 3) prange += p3;
    for (int ix = -prange; ix <= prange; ix++)
      for (int iy = -prange; iy <= prange; iy++)
        for (int iz = -prange; iz <= prange; iz++) {
          const double sh[3] = {ix * (double)cycle, iy * (double)cycle, iz * (double)cycle};
          for (int i = 0; i < nt; i++)
            for (int d = 0; d < 3; d++) xt[3 * i + d] = x0[3 * i + d] - sh[d];
          int rc = fmm_b200_direct(ctx_.cfg.device, nt, xt.data(), ns, xs.data(), qs.data(),
                                   (double)(int)ctx_.cfg.eps2, out.data());
          if (rc != FMM_OK) throw Error(rc, "direct sum failed");
          for (size_t k = 0; k < acc.size(); k++) acc[k] += out[k];
        }
    for (int i = 0; i < nt; i++)
      for (int d = 0; d < 4; d++) ibodies[i].TRG[d] += ibodies[i].SRC * acc[4 * (size_t)i + d];
  }
  void normalize(Bodies& bodies) {  // include/traversal.h:333-337
    for (Body& B : bodies)
      for (int d = 0; d < 4; d++) B.TRG[d] /= B.SRC;
  }
  void printTraversalData() {}

 private:
  Context& ctx_;
};

// namespace kernel (include/kernel.h:6-14): the translation operators one cell (pair) at
// a time, with the reference's signatures and semantics.  Each call moves the cells and
// bodies it touches to the device, runs the library's kernel for the Context's basis, order
// and precision (fmm_b200_kernel_*), and writes the results back into the host Cells and
// Bodies: M (P2M, M2M) and L (M2L, L2L) accumulate; TRG accumulates as the reference's does,
// times the target charge in P2P (LaplaceP2PCPU.cxx:151), divided by it at the start of L2P
// (LaplaceSphericalCPU.cxx:235).  Multipoles are the unnormalised ones of the reference's
// non-MASS build.  A periodic shift Xperiodic must be (ix, iy, iz) cycle with |i| <= 1, as the
// traversal forms it.  For many cells at once use the list form, fmm_b200_kernel_*.
namespace kernel {
namespace detail {

inline int nt(Context& ctx) { return nterm(ctx.cfg); }
inline int width(Context& ctx) { return ctx.cfg.basis == FMM_SPHERICAL ? 2 : 1; }

// cells uploaded for one call: bodies (x, q), cell records, M and L rows
struct Batch {
  Context& ctx;
  std::vector<double> x, q, X, R, M, L;
  std::vector<int> ibody, nbody, ichild, nchild, iparent;
  explicit Batch(Context& c) : ctx(c) {}
  int add_bodies(B_iter B, int n) {
    const int first = (int)q.size();
    for (int i = 0; i < n; i++, ++B) {
      for (int d = 0; d < 3; d++) x.push_back(B->X[d]);
      q.push_back(B->SRC);
    }
    return first;
  }
  void put(std::vector<double>& dst, const std::vector<complex_t>& e) {
    for (int t = 0; t < nt(ctx); t++) {
      const complex_t v = t < (int)e.size() ? e[t] : complex_t(0, 0);
      dst.push_back(v.real());
      if (width(ctx) == 2) dst.push_back(v.imag());
    }
  }
  int add_cell(const Cell& C, int ib, int nb, int ic = 0, int nc = 0, int ip = 0) {
    for (int d = 0; d < 3; d++) X.push_back(C.X[d]);
    R.push_back(C.R);
    ibody.push_back(ib);
    nbody.push_back(nb);
    ichild.push_back(ic);
    nchild.push_back(nc);
    iparent.push_back(ip);
    put(M, C.M);
    put(L, C.L);
    return (int)R.size() - 1;
  }
  fmm_b200_solver* upload() {
    fmm_b200_solver* h = ctx.kget();
    ctx.check(fmm_b200_set_bodies_host(h, (int)q.size(), x.data(), q.data()));
    ctx.check(fmm_b200_kernel_set_cells(h, (int)R.size(), X.data(), R.data(), ibody.data(),
                                        nbody.data(), ichild.data(), nchild.data(),
                                        iparent.data()));
    ctx.check(fmm_b200_kernel_set_expansion(h, 0, M.data()));
    ctx.check(fmm_b200_kernel_set_expansion(h, 1, L.data()));
    return h;
  }
  void fetch(int which, int cell, std::vector<complex_t>& out) {
    std::vector<double> e(M.size());
    ctx.check(fmm_b200_get_expansion(ctx.kget(), which, e.data()));
    const int w = width(ctx), n = nt(ctx);
    out.resize(n);
    for (int t = 0; t < n; t++) {
      const size_t k = ((size_t)cell * n + t) * w;
      out[t] = w == 2 ? complex_t(e[k], e[k + 1]) : complex_t(e[k], 0);
    }
  }
  std::vector<double> trg() {
    std::vector<double> t(4 * q.size());
    if (!q.empty()) ctx.check(fmm_b200_kernel_get_trg(ctx.kget(), t.data()));
    return t;
  }
};

// image code of a shift (ix, iy, iz) cycle, |i| <= 1 (the code of fmm_b200_get_lists), with
// the handle's period set to that cycle
inline int image_code(Context& ctx, const vec3& Xp) {
  double c = 0;
  for (int d = 0; d < 3; d++) c = std::max(c, Xp[d] < 0 ? -Xp[d] : Xp[d]);
  if (c == 0) return 0;
  int code = 0;
  for (int d = 0; d < 3; d++) {
    const int i = Xp[d] == 0 ? 0 : (Xp[d] == c ? 1 : (Xp[d] == -c ? 2 : -1));
    if (i < 0) throw Error(FMM_ERR_NOT_SUPPORTED, "Xperiodic must be (ix, iy, iz) * cycle");
    code = 3 * code + i;
  }
  ctx.check(fmm_b200_set_periodic(ctx.kget(), 1, c));
  return code;
}

}  // namespace detail

inline void P2M(C_iter C, Context& ctx = Context::global()) {
  detail::Batch b(ctx);
  b.add_cell(*C, b.add_bodies(C->BODY, C->NBODY), C->NBODY);
  const int c0 = 0;
  ctx.check(fmm_b200_kernel_p2m(b.upload(), 1, &c0));
  b.fetch(0, 0, C->M);
}

inline void M2M(C_iter Ci, C_iter C0, Context& ctx = Context::global()) {
  detail::Batch b(ctx);
  b.add_cell(*Ci, 0, 0, 1, Ci->NCHILD);
  for (int k = 0; k < Ci->NCHILD; k++) b.add_cell(*(C0 + Ci->ICHILD + k), 0, 0);
  const int c0 = 0;
  ctx.check(fmm_b200_kernel_m2m(b.upload(), 1, &c0));
  b.fetch(0, 0, Ci->M);
}

inline void M2L(C_iter Ci, C_iter Cj, vec3 Xperiodic, bool mutual,
                Context& ctx = Context::global()) {
  detail::Batch b(ctx);
  b.add_cell(*Ci, 0, 0);
  b.add_cell(*Cj, 0, 0);
  const int i = 0, j = 1, img = detail::image_code(ctx, Xperiodic);
  fmm_b200_solver* h = b.upload();
  ctx.check(fmm_b200_kernel_m2l(h, 1, &i, &j, &img, mutual ? 1 : 0));
  b.fetch(1, 0, Ci->L);
  if (mutual) b.fetch(1, 1, Cj->L);
}

inline void L2L(C_iter Ci, C_iter C0, Context& ctx = Context::global()) {
  detail::Batch b(ctx);
  b.add_cell(*Ci, 0, 0, 0, 0, 1);
  b.add_cell(*(C0 + Ci->IPARENT), 0, 0);
  const int c0 = 0;
  ctx.check(fmm_b200_kernel_l2l(b.upload(), 1, &c0));
  b.fetch(1, 0, Ci->L);
}

inline void L2P(C_iter Ci, Context& ctx = Context::global()) {
  detail::Batch b(ctx);
  b.add_cell(*Ci, b.add_bodies(Ci->BODY, Ci->NBODY), Ci->NBODY);
  fmm_b200_solver* h = b.upload();
  std::vector<double> t(4 * (size_t)Ci->NBODY);
  B_iter B = Ci->BODY;
  for (int k = 0; k < Ci->NBODY; k++, ++B)
    for (int d = 0; d < 4; d++) t[4 * k + d] = B->TRG[d] / B->SRC;  // TRG /= SRC first
  ctx.check(fmm_b200_kernel_set_trg(h, t.data()));
  const int c0 = 0;
  ctx.check(fmm_b200_kernel_l2p(h, 1, &c0));
  t = b.trg();
  B = Ci->BODY;
  for (int k = 0; k < Ci->NBODY; k++, ++B)
    for (int d = 0; d < 4; d++) B->TRG[d] = t[4 * k + d];
}

inline void P2P(C_iter Ci, C_iter Cj, real_t eps2, vec3 Xperiodic, bool mutual,
                Context& ctx = Context::global()) {
  detail::Batch b(ctx);
  b.add_cell(*Ci, b.add_bodies(Ci->BODY, Ci->NBODY), Ci->NBODY);
  b.add_cell(*Cj, b.add_bodies(Cj->BODY, Cj->NBODY), Cj->NBODY);
  const int i = 0, j = 1, img = detail::image_code(ctx, Xperiodic);
  ctx.check(fmm_b200_kernel_p2p(b.upload(), 1, &i, &j, &img, mutual ? 1 : 0, (double)eps2));
  const std::vector<double> t = b.trg();
  B_iter B = Ci->BODY;
  for (int k = 0; k < Ci->NBODY; k++, ++B)
    for (int d = 0; d < 4; d++) B->TRG[d] += B->SRC * t[4 * k + d];
  if (mutual) {
    B = Cj->BODY;
    for (int k = 0; k < Cj->NBODY; k++, ++B)
      for (int d = 0; d < 4; d++) B->TRG[d] += B->SRC * t[4 * (Ci->NBODY + k) + d];
  }
}

inline void P2P(C_iter C, real_t eps2, Context& ctx = Context::global()) {
  detail::Batch b(ctx);
  b.add_cell(*C, b.add_bodies(C->BODY, C->NBODY), C->NBODY);
  const int c0 = 0;
  ctx.check(fmm_b200_kernel_p2p(b.upload(), 1, &c0, &c0, nullptr, 0, (double)eps2));
  const std::vector<double> t = b.trg();
  B_iter B = C->BODY;
  for (int k = 0; k < C->NBODY; k++, ++B)
    for (int d = 0; d < 4; d++) B->TRG[d] += B->SRC * t[4 * k + d];
}

}  // namespace kernel

// Verify (include/verify.h:18-83)
struct Verify {
  double getDifScalar(const Bodies& a, const Bodies& b) const {
    double v = 0;
    for (size_t i = 0; i < a.size(); i++) v += (a[i].TRG[0] - b[i].TRG[0]) * (a[i].TRG[0] - b[i].TRG[0]);
    return v;
  }
  double getNrmScalar(const Bodies& a) const {
    double v = 0;
    for (const Body& B : a) v += B.TRG[0] * B.TRG[0];
    return v;
  }
  double getDifVector(const Bodies& a, const Bodies& b) const {
    double v = 0;
    for (size_t i = 0; i < a.size(); i++)
      for (int d = 1; d < 4; d++) v += (a[i].TRG[d] - b[i].TRG[d]) * (a[i].TRG[d] - b[i].TRG[d]);
    return v;
  }
  double getNrmVector(const Bodies& a) const {
    double v = 0;
    for (const Body& B : a)
      for (int d = 1; d < 4; d++) v += B.TRG[d] * B.TRG[d];
    return v;
  }
};

}  // namespace exafmm_b200
