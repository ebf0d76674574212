// The examples/kernel.cxx sequence written against namespace kernel of
// include/exafmm_b200.hpp: 16 sources in a cell at (1,1,1), P2M -> M2M into its parent at
// the origin -> M2L into a cell at R + 4 -> L2L into its child at R + 3 -> L2P at 16
// targets, against P2P of the same targets and sources (then TRG / SRC); theta = 0.5,
// R = 2 / theta, positions and charges from drand48 in its unseeded state, as a fresh
// kernel.cxx process draws them.  Prints "<P> <rel-L2 error of the potential>".
// Usage: kernel_example <spherical|cartesian> <P> [f32|f64]
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "exafmm_b200.hpp"

using namespace exafmm_b200;

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: kernel_example <spherical|cartesian> <P> [f32|f64]\n");
    return 2;
  }
  Context& ctx = Context::global();
  ctx.cfg.basis = std::strcmp(argv[1], "cartesian") == 0 ? FMM_CARTESIAN : FMM_SPHERICAL;
  ctx.cfg.P = std::atoi(argv[2]);
  ctx.cfg.precision = argc > 3 && std::strcmp(argv[3], "f32") == 0 ? FMM_FP32 : FMM_FP64;
  const double theta = 0.5, R = 2 / theta;
  Bodies sources(16), targets(16), direct(16);
  Cells cells(4);
  const vec3 none;
  try {
    for (Body& B : sources) {
      for (int d = 0; d < 3; d++) B.X[d] = 2 * drand48();
      B.SRC = drand48();
    }
    C_iter Cj = cells.begin(), CJ = cells.begin() + 1, CI = cells.begin() + 2,
           Ci = cells.begin() + 3;
    for (int d = 0; d < 3; d++) {
      Cj->X[d] = 1;
      CJ->X[d] = 0;
      CI->X[d] = R + 4;
      Ci->X[d] = R + 3;
    }
    Cj->BODY = sources.begin();
    Cj->NBODY = 16;
    kernel::P2M(Cj);
    CJ->ICHILD = 0;
    CJ->NCHILD = 1;
    kernel::M2M(CJ, cells.begin());
    kernel::M2L(CI, CJ, none, false);
    Ci->IPARENT = 2;
    kernel::L2L(Ci, cells.begin());
    for (Body& B : targets) {
      for (int d = 0; d < 3; d++) B.X[d] = R + 2 + 2 * drand48();
      B.SRC = drand48();
    }
    Ci->BODY = targets.begin();
    Ci->NBODY = 16;
    kernel::L2P(Ci);
    for (int b = 0; b < 16; b++) {
      direct[b] = targets[b];
      for (int d = 0; d < 4; d++) direct[b].TRG[d] = 0;
    }
    Ci->BODY = direct.begin();
    kernel::P2P(Ci, Cj, 0.0, none, false);
    double diff = 0, norm = 0;
    for (int b = 0; b < 16; b++) {
      const double d = direct[b].TRG[0] / direct[b].SRC;
      diff += (targets[b].TRG[0] - d) * (targets[b].TRG[0] - d);
      norm += d * d;
    }
    std::printf("%d %.10e\n", ctx.cfg.P, std::sqrt(diff / norm));
  } catch (const Error& e) {
    std::fprintf(stderr, "error %d: %s\n", e.code, e.what());
    return 1;
  }
  return 0;
}
