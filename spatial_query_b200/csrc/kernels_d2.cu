// Kernel instantiations for D = 2 (one translation unit per dimension so
// they compile in parallel).
#include "traverse.cuh"

namespace sq {
bool kernel_set_d2(int narrow, KernelSet* out) {
  switch (narrow) {
    case kNarrowAabb: *out = make_kernel_set<2, kNarrowAabb>(); return true;
    case kNarrowSphere: *out = make_kernel_set<2, kNarrowSphere>(); return true;
    case kNarrowSphereNear: *out = make_kernel_set<2, kNarrowSphereNear>(); return true;
    default: return false;
  }
}
}  // namespace sq
