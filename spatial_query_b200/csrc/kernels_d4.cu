// Kernel instantiations for D = 4 (one translation unit per dimension so
// they compile in parallel).
#include "traverse.cuh"

namespace sq {
bool kernel_set_d4(int narrow, KernelSet* out) {
  switch (narrow) {
    case kNarrowAabb: *out = make_kernel_set<4, kNarrowAabb>(); return true;
    case kNarrowSphere: *out = make_kernel_set<4, kNarrowSphere>(); return true;
    case kNarrowSphereNear: *out = make_kernel_set<4, kNarrowSphereNear>(); return true;
    default: return false;
  }
}
}  // namespace sq
