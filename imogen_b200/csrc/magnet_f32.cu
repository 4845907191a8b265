// Magnet sweep kernels in float: the launch entry points of sweeps.cuh for this precision.
#include "sweeps_impl.cuh"

namespace img {
template cudaError_t launch_mag_chain<float>(const MagArgs&, const PencilLaunch&);
template cudaError_t launch_mag_chain_batch<float>(const MagArgs*, const BlockMap*, const PencilLaunch&);
template cudaError_t launch_mag_ctcell_batch<float>(const MagArgs*, const BlockMap*, const PencilLaunch&);
template cudaError_t launch_mag_ctcell<float>(const MagArgs&, const PencilLaunch&);
template cudaError_t chain_attributes<float>(int, int);
}  // namespace img
