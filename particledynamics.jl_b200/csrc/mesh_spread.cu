// Spread launchers of the mesh engine (B-spline and prolate windows, orders 3..12).
// One translation unit per launcher family, so that the kernel variants compile in parallel.
#include "mesh_kernels.cuh"

namespace pdb {

PD_SPREAD_LAUNCHER(WIN_BSPLINE);
PD_SPREAD_LAUNCHER(WIN_PROLATE);

}  // namespace pdb
