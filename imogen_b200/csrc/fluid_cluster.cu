// Batched fluid sweeps over pencils that span a thread-block cluster (both precisions).
//
// This translation unit is compiled with -Xptxas -O1 (imogen_b200/build.py).  At the default -O3 the
// batched form of the halo-job fluid kernel (fade boundaries, 4 cells per thread, 4-CTA clusters,
// FP32) computed garbage pencil maxima, while the same kernel body launched alone matched the oracle;
// compiled at -O1 the batched form matches the oracle and the launch alone.  The cause was not
// identified, so the batched cluster launches of every variant and precision use the kernel template
// below, which is instantiated in this unit only (a kernel template instantiated in two units would
// share one host stub and could launch the other unit's copy).  They run only for pencils longer than
// one CTA; cluster tilings never take the copy-ghost variants.
#include "sweeps_impl.cuh"

namespace img {

template <typename T, bool MHD, int CPT, int V>
__global__ void __launch_bounds__(512, CPT == 1 ? 2 : 1) fluid_sweep_cluster_batch_kernel(
    const FluidArgs* __restrict__ args, const BlockMap* __restrict__ map) {
    __shared__ FluidArgs sa;
    const BlockMap bm = map[blockIdx.x];
    load_member_args(sa, args + bm.member);
    __syncthreads();
    fluid_sweep_body<T, MHD, CPT, V>(sa, (unsigned)bm.block);
}

template <typename T, bool MHD, int V>
void (*cluster_kernel_cpt(int cpt))(const FluidArgs*, const BlockMap*) {
    switch (cpt) {
        case 1: return fluid_sweep_cluster_batch_kernel<T, MHD, 1, V>;
        case 2: return fluid_sweep_cluster_batch_kernel<T, MHD, 2, V>;
        default: return fluid_sweep_cluster_batch_kernel<T, MHD, 4, V>;
    }
}

// variants of cluster tilings: 0 halo jobs, 1 with fade, 3 and 4 the stored-edge capturing forms
template <typename T, bool MHD>
void (*cluster_kernel_v(int cpt, int v))(const FluidArgs*, const BlockMap*) {
    switch (v) {
        case 1: return cluster_kernel_cpt<T, MHD, 1>(cpt);
        case 3: return cluster_kernel_cpt<T, MHD, 3>(cpt);
        case 4: return cluster_kernel_cpt<T, MHD, 4>(cpt);
        default: return cluster_kernel_cpt<T, MHD, 0>(cpt);
    }
}

template <typename T>
void (*cluster_kernel(int cpt, bool mhd, int v))(const FluidArgs*, const BlockMap*) {
    return mhd ? cluster_kernel_v<T, true>(cpt, v) : cluster_kernel_v<T, false>(cpt, v);
}

template <typename T>
cudaError_t launch_fluid_sweep_batch_cluster(const FluidArgs* args, const BlockMap* map, const PencilLaunch& L,
                                             bool mhd) {
    if (L.cg) return cudaErrorInvalidConfiguration;   // copy ghosts need single-CTA pencils
    return launch_pencil_batch(cluster_kernel<T>(L.cpt, mhd, kernel_variant(L.fade, L.cg, L.init)), args, map, L);
}

template <typename T>
cudaError_t fluid_cluster_attributes(int cpt, int optin) {
    for (int mhd = 0; mhd < 2; ++mhd)
        for (int v : {0, 1, 3, 4}) {
            cudaError_t e = allow_max_smem(cluster_kernel<T>(cpt, mhd != 0, v), optin);
            if (e != cudaSuccess) return e;
        }
    return cudaSuccess;
}

template cudaError_t launch_fluid_sweep_batch_cluster<float>(const FluidArgs*, const BlockMap*, const PencilLaunch&, bool);
template cudaError_t launch_fluid_sweep_batch_cluster<double>(const FluidArgs*, const BlockMap*, const PencilLaunch&, bool);
template cudaError_t fluid_cluster_attributes<float>(int, int);
template cudaError_t fluid_cluster_attributes<double>(int, int);

}  // namespace img
