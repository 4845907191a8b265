// Definitions of the launch entry points declared in sweeps.cuh.  Each translation unit that
// includes this file instantiates them for one precision.
#pragma once

#include "sweeps.cuh"

namespace img {

template <typename Args>
cudaError_t launch_pencil(void (*kern)(const Args), const Args& a, const PencilLaunch& L) {
    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(L.grid_x, L.grid_y);
    lc.blockDim = dim3(L.block);
    lc.dynamicSmemBytes = L.smem;
    lc.stream = L.stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = L.cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    return cudaLaunchKernelEx(&lc, kern, a);
}

template <typename T, bool MHD, bool FADE>
void (*fluid_kernel(int cpt))(const FluidArgs) {
    switch (cpt) {
        case 1: return fluid_sweep_kernel<T, MHD, 1, FADE>;
        case 2: return fluid_sweep_kernel<T, MHD, 2, FADE>;
        default: return fluid_sweep_kernel<T, MHD, 4, FADE>;
    }
}

template <typename T, bool FADE>
void (*chain_kernel(int cpt))(const MagArgs) {
    switch (cpt) {
        case 1: return mag_chain_kernel<T, 1, FADE>;
        case 2: return mag_chain_kernel<T, 2, FADE>;
        default: return mag_chain_kernel<T, 4, FADE>;
    }
}

template <typename T>
void (*fluid_kernel(int cpt, bool mhd, bool fade))(const FluidArgs) {
    if (mhd) return fade ? fluid_kernel<T, true, true>(cpt) : fluid_kernel<T, true, false>(cpt);
    return fade ? fluid_kernel<T, false, true>(cpt) : fluid_kernel<T, false, false>(cpt);
}

template <typename T>
cudaError_t launch_fluid_sweep(const FluidArgs& a, const PencilLaunch& L, bool mhd) {
    return launch_pencil(fluid_kernel<T>(L.cpt, mhd, L.fade), a, L);
}

template <typename T>
cudaError_t launch_mag_chain(const MagArgs& a, const PencilLaunch& L) {
    return launch_pencil(L.fade ? chain_kernel<T, true>(L.cpt) : chain_kernel<T, false>(L.cpt), a, L);
}

template <typename T>
cudaError_t launch_mag_ct(const MagArgs& a, unsigned blocks, cudaStream_t stream) {
    mag_ct_kernel<T><<<blocks, 256, 0, stream>>>(a);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_mag_cell(const MagArgs& a, unsigned blocks, cudaStream_t stream) {
    mag_cell_kernel<T><<<blocks, 256, 0, stream>>>(a);
    return cudaGetLastError();
}

template <typename T>
cudaError_t fluid_attributes(int cpt, size_t smem) {
    for (int v = 0; v < 4; ++v) {
        cudaError_t e = cudaFuncSetAttribute(fluid_kernel<T>(cpt, v & 1, v >> 1),
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <typename T>
cudaError_t chain_attributes(int cpt, size_t smem) {
    for (int v = 0; v < 2; ++v) {
        cudaError_t e = cudaFuncSetAttribute(v ? chain_kernel<T, true>(cpt) : chain_kernel<T, false>(cpt),
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <typename T>
cudaError_t fluid_max_clusters(const PencilLaunch& L, int* n) {
    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(L.cluster);
    lc.blockDim = dim3(L.block);
    lc.dynamicSmemBytes = L.smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = L.cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    return cudaOccupancyMaxActiveClusters(n, fluid_kernel<T>(L.cpt, true, L.fade), &lc);
}

}  // namespace img
