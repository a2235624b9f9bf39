// AD gather of the B-spline mesh joined with the slot pair forces and the closing kick (the step).
// One translation unit per launcher family, so that the kernel variants compile in parallel.
#include "mesh_kernels.cuh"

namespace pdb {

PD_GATHER_LAUNCHER(WIN_BSPLINE, false, 2);

}  // namespace pdb
