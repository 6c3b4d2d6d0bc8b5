// Two-level kernel instantiations: meshes at D = 3, oriented boxes and balls
// at D = 2, 3, 4 and 6.
#include "tlas.cuh"

namespace sq {
bool tlas_kernel_set(int dim, int kind, TlasKernelSet* out) {
  switch (dim * 16 + kind) {
    case 3 * 16 + kInstMesh: *out = make_tlas_kernel_set<3, kInstMesh>(); return true;
    case 3 * 16 + kInstBox: *out = make_tlas_kernel_set<3, kInstBox>(); return true;
    case 3 * 16 + kInstBall: *out = make_tlas_kernel_set<3, kInstBall>(); return true;
    case 2 * 16 + kInstBox: *out = make_tlas_kernel_set<2, kInstBox>(); return true;
    case 2 * 16 + kInstBall: *out = make_tlas_kernel_set<2, kInstBall>(); return true;
    case 4 * 16 + kInstBox: *out = make_tlas_kernel_set<4, kInstBox>(); return true;
    case 4 * 16 + kInstBall: *out = make_tlas_kernel_set<4, kInstBall>(); return true;
    case 6 * 16 + kInstBox: *out = make_tlas_kernel_set<6, kInstBox>(); return true;
    case 6 * 16 + kInstBall: *out = make_tlas_kernel_set<6, kInstBall>(); return true;
    default: return false;
  }
}
}  // namespace sq
