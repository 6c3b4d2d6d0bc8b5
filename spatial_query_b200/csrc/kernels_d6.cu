// Kernel instantiations for D = 6 (one translation unit per dimension so
// they compile in parallel).
#include "traverse.cuh"

namespace sq {
bool kernel_set_d6(int narrow, KernelSet* out) {
  switch (narrow) {
    case kNarrowAabb: *out = make_kernel_set<6, kNarrowAabb>(); return true;
    case kNarrowSphere: *out = make_kernel_set<6, kNarrowSphere>(); return true;
    case kNarrowSphereNear: *out = make_kernel_set<6, kNarrowSphereNear>(); return true;
    default: return false;
  }
}
}  // namespace sq
