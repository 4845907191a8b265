// Fluid sweep kernels in double: the launch entry points of sweeps.cuh for this precision.
#include "sweeps_impl.cuh"

namespace img {
template cudaError_t launch_fluid_sweep<double>(const FluidArgs&, const PencilLaunch&, bool);
template cudaError_t launch_fluid_sweep_batch<double>(const FluidArgs*, const BlockMap*, const PencilLaunch&, bool);
template cudaError_t fluid_attributes<double>(int, int);
template cudaError_t fluid_max_clusters<double>(const PencilLaunch&, int*);
template cudaError_t fluid_seg_attributes<double>(int);
}  // namespace img
