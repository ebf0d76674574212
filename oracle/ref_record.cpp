// Test infrastructure only: stands in for namespace kernel (include/kernel.h:6-14) in the
// reference harness, records which cell pairs the dual-tree traversal hands to M2L and P2P
// (include/traversal.h:41,52,54), and forwards every call to the reference kernels, which
// oracle/Makefile compiles with -Dkernel=refkernel.
#define kernel refkernel
#include "kernel.h"
#undef kernel
#undef kernel_h
#include "kernel.h"
#include <vector>

namespace refrec {
bool enabled = false;
C_iter Ci0, Cj0;
std::vector<long long> m2l, p2p;
static inline long long pack(C_iter Ci, C_iter Cj) {
  return ((long long)(Ci - Ci0) << 32) | (long long)(Cj - Cj0);
}
}  // namespace refrec

void kernel::P2P(C_iter Ci, C_iter Cj, real_t eps2, vec3 Xperiodic, bool mutual) {
  if (refrec::enabled) refrec::p2p.push_back(refrec::pack(Ci, Cj));
  refkernel::P2P(Ci, Cj, eps2, Xperiodic, mutual);
}
void kernel::P2P(C_iter C, real_t eps2) {
  if (refrec::enabled) refrec::p2p.push_back(refrec::pack(C, C));
  refkernel::P2P(C, eps2);
}
void kernel::P2M(C_iter C) { refkernel::P2M(C); }
void kernel::M2M(C_iter Ci, C_iter C0) { refkernel::M2M(Ci, C0); }
void kernel::M2L(C_iter Ci, C_iter Cj, vec3 Xperiodic, bool mutual) {
  if (refrec::enabled) refrec::m2l.push_back(refrec::pack(Ci, Cj));
  refkernel::M2L(Ci, Cj, Xperiodic, mutual);
}
void kernel::L2L(C_iter Ci, C_iter C0) { refkernel::L2L(Ci, C0); }
void kernel::L2P(C_iter Ci) { refkernel::L2P(Ci); }
