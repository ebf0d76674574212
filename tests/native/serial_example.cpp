// The examples/serial.cxx:41-84 sequence written against include/exafmm_b200.hpp: FMM on
// the GPU, then Traversal::direct on stride-sampled targets and the rel-L2 errors of
// potential and acceleration.  Prints "pot <err> acc <err>"; exit status 0 when both are
// below 1e-3.  Usage: serial_example [N]
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>

#include "exafmm_b200.hpp"

using namespace exafmm_b200;

int main(int argc, char** argv) {
  const int N = argc > 1 ? std::atoi(argv[1]) : 20000;
  Context& ctx = Context::global();
  ctx.cfg.P = 8;
  Bodies bodies(N), buffer;
  std::mt19937_64 rng(1);
  std::uniform_real_distribution<double> u(-1, 1);
  double avg = 0;
  for (int i = 0; i < N; i++) {
    for (int d = 0; d < 3; d++) bodies[i].X[d] = u(rng);
    bodies[i].SRC = u(rng);
    bodies[i].IBODY = i;
    avg += bodies[i].SRC;
  }
  for (Body& B : bodies) B.SRC -= avg / N;
  BoundBox boundBox(1000);
  BuildTree buildTree(64, 1000);
  UpDownPass upDownPass(0.4, true, false);
  Traversal traversal(1000, 0, 0.0);
  try {
    Bounds bounds = boundBox.getBounds(bodies);
    Cells cells = buildTree.buildTree(bodies, buffer, bounds);
    upDownPass.upwardPass(cells);
    traversal.dualTreeTraversal(cells, cells, 2 * M_PI, false);
    upDownPass.downwardPass(cells);
    // Dataset::sampleBodies (include/dataset.h:268-276) + direct + normalize
    const int nt = 100, stride = N / nt;
    Bodies targets(nt), fmm(nt);
    for (int i = 0; i < nt; i++) {
      fmm[i] = bodies[i * stride];
      targets[i] = bodies[i * stride];
      targets[i].TRG = vec4();
    }
    traversal.direct(targets, bodies, 2 * M_PI);
    traversal.normalize(targets);
    Verify v;
    double pot = std::sqrt(v.getDifScalar(fmm, targets) / v.getNrmScalar(targets));
    double acc = std::sqrt(v.getDifVector(fmm, targets) / v.getNrmVector(targets));
    std::printf("cells %zu pot %.3e acc %.3e\n", cells.size(), pot, acc);
    return pot < 1e-3 && acc < 1e-3 ? 0 : 1;
  } catch (const Error& e) {
    std::printf("error %d: %s\n", e.code, e.what());
    return 2;
  }
}
