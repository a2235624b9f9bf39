// ik gather of the B-spline mesh (P3M-ik) joined with the slot pair forces and the closing kick.
// One translation unit per launcher family, so that the kernel variants compile in parallel.
#include "mesh_kernels.cuh"

namespace pdb {

PD_GATHER_LAUNCHER(WIN_BSPLINE, true, 2);

}  // namespace pdb
