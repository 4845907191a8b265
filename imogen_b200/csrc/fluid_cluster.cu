// Batched fluid sweeps over pencils that span a thread-block cluster (both precisions).
//
// This translation unit is compiled with -Xptxas -O1 (imogen_b200/build.py).  At the default -O3 the
// batched form of the halo-job fluid kernel with fade boundaries, 4 cells per thread and 4-CTA
// clusters (FP32) computed garbage pencil maxima, while the same kernel body launched alone was
// correct; the same source compiled at -O1 gives results bitwise equal to the launches alone.  The
// cause was not identified, so the batched cluster launches of every variant and precision are kept
// here, away from the -O3 code.  They run only for pencils longer than one CTA.
#include "sweeps_impl.cuh"

namespace img {

template <typename T>
cudaError_t launch_fluid_sweep_batch_cluster(const FluidArgs* args, const BlockMap* map, const PencilLaunch& L,
                                             bool mhd) {
    return launch_pencil_batch(fluid_batch_kernel<T>(L.cpt, mhd, kernel_variant(L.fade, L.cg, L.init)), args, map, L);
}

template <typename T>
cudaError_t fluid_cluster_attributes(int cpt, int optin) {
    for (int v = 0; v < 12; ++v) {
        cudaError_t e = allow_max_smem(fluid_batch_kernel<T>(cpt, v & 1, v >> 1), optin);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template cudaError_t launch_fluid_sweep_batch_cluster<float>(const FluidArgs*, const BlockMap*, const PencilLaunch&, bool);
template cudaError_t launch_fluid_sweep_batch_cluster<double>(const FluidArgs*, const BlockMap*, const PencilLaunch&, bool);
template cudaError_t fluid_cluster_attributes<float>(int, int);
template cudaError_t fluid_cluster_attributes<double>(int, int);

}  // namespace img
