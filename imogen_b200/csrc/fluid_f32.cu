// Fluid sweep kernels in float: the launch entry points of sweeps.cuh for this precision.
#include "sweeps_impl.cuh"

namespace img {
template cudaError_t launch_fluid_sweep<float>(const FluidArgs&, const PencilLaunch&, bool);
template cudaError_t launch_fluid_sweep_batch<float>(const FluidArgs*, const BlockMap*, const PencilLaunch&, bool);
template cudaError_t fluid_attributes<float>(int, int);
template cudaError_t fluid_max_clusters<float>(const PencilLaunch&, int*);
template cudaError_t fluid_seg_attributes<float>(int);
}  // namespace img
