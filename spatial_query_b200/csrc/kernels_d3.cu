// Kernel instantiations for D = 3 (one translation unit per dimension so
// they compile in parallel).
#include "traverse.cuh"

namespace sq {
bool kernel_set_d3(int narrow, KernelSet* out) {
  switch (narrow) {
    case kNarrowAabb: *out = make_kernel_set<3, kNarrowAabb>(); return true;
    case kNarrowSphere: *out = make_kernel_set<3, kNarrowSphere>(); return true;
    case kNarrowSphereNear: *out = make_kernel_set<3, kNarrowSphereNear>(); return true;
    case kNarrowTri: *out = make_kernel_set<3, kNarrowTri>(); return true;
    default: return false;
  }
}
}  // namespace sq
