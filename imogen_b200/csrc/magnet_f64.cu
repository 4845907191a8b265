// Magnet sweep kernels in double: the launch entry points of sweeps.cuh for this precision.
#include "sweeps_impl.cuh"

namespace img {
template cudaError_t launch_mag_chain<double>(const MagArgs&, const PencilLaunch&);
template cudaError_t launch_mag_chain_batch<double>(const MagArgs*, const BlockMap*, const PencilLaunch&);
template cudaError_t launch_mag_ctcell_batch<double>(const MagArgs*, const BlockMap*, const PencilLaunch&);
template cudaError_t launch_mag_ctcell<double>(const MagArgs&, const PencilLaunch&);
template cudaError_t chain_attributes<double>(int, int);
}  // namespace img
