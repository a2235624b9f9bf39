// AD gathers of the prolate-window mesh (ESP), add and set modes (pd_mesh_gather).
// One translation unit per launcher family, so that the kernel variants compile in parallel.
#include "mesh_kernels.cuh"

namespace pdb {

PD_GATHER_LAUNCHER(WIN_PROLATE, false, 0);
PD_GATHER_LAUNCHER(WIN_PROLATE, false, 1);

}  // namespace pdb
