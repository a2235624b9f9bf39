// ik gathers of the B-spline mesh (P3M-ik), add and set modes (pd_mesh_gather).
// One translation unit per launcher family, so that the kernel variants compile in parallel.
#include "mesh_kernels.cuh"

namespace pdb {

PD_GATHER_LAUNCHER(WIN_BSPLINE, true, 0);
PD_GATHER_LAUNCHER(WIN_BSPLINE, true, 1);

}  // namespace pdb
