// Test infrastructure only: stands in for namespace kernel (include/kernel.h:6-14) in the
// reference harness, records which cell pairs the dual-tree traversal hands to M2L and P2P
// (include/traversal.h:41,52,54), and forwards every call to the reference kernels, which
// oracle/Makefile compiles with -Dkernel=refkernel.
#define kernel refkernel
#include "kernel.h"
#undef kernel
#undef kernel_h
#include "kernel.h"
#include <cmath>
#include <cstdint>
#include <vector>

namespace refrec {
bool enabled = false;
C_iter Ci0, Cj0;
long long ncells = 0;
double cycle = 1;
std::vector<long long> m2l, p2p;
// image code of a shift of (ix, iy, iz) periods, |i| <= 1: 9 d(ix) + 3 d(iy) + d(iz) with
// d(0) = 0, d(1) = 1, d(-1) = 2
static inline long long image(const vec3& Xp) {
  long long c = 0;
  for (int d = 0; d < 3; d++) {
    const long i = std::lround(Xp[d] / cycle);
    c = 3 * c + (i < 0 ? 2 : i);
  }
  return c;
}
// by address: iterator subtraction across unrelated arrays is undefined (compilers divide
// the byte distance by sizeof(Cell) assuming it is a multiple of it)
static inline bool in_tree(C_iter C) {
  const std::uintptr_t a = reinterpret_cast<std::uintptr_t>(&*C);
  const std::uintptr_t b = reinterpret_cast<std::uintptr_t>(&*Cj0);
  return a >= b && a < b + (std::uintptr_t)ncells * sizeof(Cell);
}
static inline long long pack(C_iter Ci, C_iter Cj, const vec3& Xp) {
  return ((long long)(Ci - Ci0) << 32) | (long long)(Cj - Cj0) | (image(Xp) << 27);
}
}  // namespace refrec

void kernel::P2P(C_iter Ci, C_iter Cj, real_t eps2, vec3 Xperiodic, bool mutual) {
  if (refrec::enabled) refrec::p2p.push_back(refrec::pack(Ci, Cj, Xperiodic));
  refkernel::P2P(Ci, Cj, eps2, Xperiodic, mutual);
}
void kernel::P2P(C_iter C, real_t eps2) {
  if (refrec::enabled) refrec::p2p.push_back(refrec::pack(C, C, vec3(0)));
  refkernel::P2P(C, eps2);
}
void kernel::P2M(C_iter C) { refkernel::P2M(C); }
void kernel::M2M(C_iter Ci, C_iter C0) { refkernel::M2M(Ci, C0); }
void kernel::M2L(C_iter Ci, C_iter Cj, vec3 Xperiodic, bool mutual) {
  if (refrec::enabled && refrec::in_tree(Cj)) refrec::m2l.push_back(refrec::pack(Ci, Cj, Xperiodic));
  refkernel::M2L(Ci, Cj, Xperiodic, mutual);
}
void kernel::L2L(C_iter Ci, C_iter C0) { refkernel::L2L(Ci, C0); }
void kernel::L2P(C_iter Ci) { refkernel::L2P(Ci); }
