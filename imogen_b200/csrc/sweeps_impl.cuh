// Definitions of the launch entry points declared in sweeps.cuh.  Each translation unit that
// includes this file instantiates them for one precision.
#pragma once

#include "sweeps.cuh"

namespace img {

inline cudaLaunchConfig_t pencil_config(const PencilLaunch& L, cudaLaunchAttribute* attr) {
    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(L.grid_x, L.grid_y);
    lc.blockDim = dim3(L.block);
    lc.dynamicSmemBytes = L.smem;
    lc.stream = L.stream;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = L.cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    return lc;
}

template <typename Args>
cudaError_t launch_pencil_batch(void (*kern)(const Args*, const BlockMap*), const Args* args, const BlockMap* map,
                                const PencilLaunch& L) {
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t lc = pencil_config(L, attr);
    return cudaLaunchKernelEx(&lc, kern, args, map);
}

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

template <typename T, bool MHD, bool FADE, bool CG>
void (*fluid_kernel(int cpt))(const FluidArgs) {
    switch (cpt) {
        case 1: return fluid_sweep_kernel<T, MHD, 1, FADE, CG>;
        case 2: return fluid_sweep_kernel<T, MHD, 2, FADE, CG>;
        default: return fluid_sweep_kernel<T, MHD, 4, FADE, CG>;
    }
}

template <typename T, bool FADE, bool CG>
void (*chain_kernel(int cpt, int nqc))(const MagArgs) {
    if (nqc == 2) return cpt == 1 ? mag_chain_kernel<T, 1, FADE, 2, CG> : mag_chain_kernel<T, 2, FADE, 2, CG>;
    switch (cpt) {
        case 1: return mag_chain_kernel<T, 1, FADE, 1, CG>;
        case 2: return mag_chain_kernel<T, 2, FADE, 1, CG>;
        default: return mag_chain_kernel<T, 4, FADE, 1, CG>;
    }
}

// Ghost variant: 0 halo jobs, 1 halo jobs with fade damping, 2 copy ghosts.
inline int ghost_variant(bool fade, bool cg) { return fade ? 1 : (cg ? 2 : 0); }

template <typename T>
void (*chain_kernel(int cpt, int nqc, int gv))(const MagArgs) {
    return gv == 1 ? chain_kernel<T, true, false>(cpt, nqc)
                   : (gv == 2 ? chain_kernel<T, false, true>(cpt, nqc) : chain_kernel<T, false, false>(cpt, nqc));
}

template <typename T, bool MHD, bool FADE, bool CG>
void (*fluid_batch_kernel(int cpt))(const FluidArgs*, const BlockMap*) {
    switch (cpt) {
        case 1: return fluid_sweep_batch_kernel<T, MHD, 1, FADE, CG>;
        case 2: return fluid_sweep_batch_kernel<T, MHD, 2, FADE, CG>;
        default: return fluid_sweep_batch_kernel<T, MHD, 4, FADE, CG>;
    }
}

template <typename T, bool FADE, bool CG>
void (*chain_batch_kernel(int cpt, int nqc))(const MagArgs*, const BlockMap*) {
    if (nqc == 2) return cpt == 1 ? mag_chain_batch_kernel<T, 1, FADE, 2, CG> : mag_chain_batch_kernel<T, 2, FADE, 2, CG>;
    switch (cpt) {
        case 1: return mag_chain_batch_kernel<T, 1, FADE, 1, CG>;
        case 2: return mag_chain_batch_kernel<T, 2, FADE, 1, CG>;
        default: return mag_chain_batch_kernel<T, 4, FADE, 1, CG>;
    }
}

template <typename T>
void (*chain_batch_kernel(int cpt, int nqc, int gv))(const MagArgs*, const BlockMap*) {
    return gv == 1 ? chain_batch_kernel<T, true, false>(cpt, nqc)
                   : (gv == 2 ? chain_batch_kernel<T, false, true>(cpt, nqc) : chain_batch_kernel<T, false, false>(cpt, nqc));
}

template <typename T>
void (*fluid_batch_kernel(int cpt, bool mhd, int gv))(const FluidArgs*, const BlockMap*) {
    if (mhd)
        return gv == 1 ? fluid_batch_kernel<T, true, true, false>(cpt)
                       : (gv == 2 ? fluid_batch_kernel<T, true, false, true>(cpt) : fluid_batch_kernel<T, true, false, false>(cpt));
    return gv == 1 ? fluid_batch_kernel<T, false, true, false>(cpt)
                   : (gv == 2 ? fluid_batch_kernel<T, false, false, true>(cpt) : fluid_batch_kernel<T, false, false, false>(cpt));
}

template <typename T>
cudaError_t launch_fluid_sweep_batch(const FluidArgs* args, const BlockMap* map, const PencilLaunch& L, bool mhd) {
    return launch_pencil_batch(fluid_batch_kernel<T>(L.cpt, mhd, ghost_variant(L.fade, L.cg)), args, map, L);
}

template <typename T>
cudaError_t launch_mag_chain_batch(const MagArgs* args, const BlockMap* map, const PencilLaunch& L) {
    return launch_pencil_batch(chain_batch_kernel<T>(L.cpt, L.nqc, ghost_variant(L.fade, L.cg)), args, map, L);
}

template <typename T, bool FADE, bool CG>
void (*ctcell_kernel(int cpt))(const MagArgs) {
    switch (cpt) {
        case 1: return mag_ctcell_kernel<T, 1, FADE, CG>;
        case 2: return mag_ctcell_kernel<T, 2, FADE, CG>;
        default: return mag_ctcell_kernel<T, 4, FADE, CG>;
    }
}

template <typename T, bool FADE, bool CG>
void (*ctcell_batch_kernel(int cpt))(const MagArgs*, const BlockMap*) {
    switch (cpt) {
        case 1: return mag_ctcell_batch_kernel<T, 1, FADE, CG>;
        case 2: return mag_ctcell_batch_kernel<T, 2, FADE, CG>;
        default: return mag_ctcell_batch_kernel<T, 4, FADE, CG>;
    }
}

template <typename T>
void (*ctcell_kernel(int cpt, int gv))(const MagArgs) {
    return gv == 1 ? ctcell_kernel<T, true, false>(cpt)
                   : (gv == 2 ? ctcell_kernel<T, false, true>(cpt) : ctcell_kernel<T, false, false>(cpt));
}

template <typename T>
void (*ctcell_batch_kernel(int cpt, int gv))(const MagArgs*, const BlockMap*) {
    return gv == 1 ? ctcell_batch_kernel<T, true, false>(cpt)
                   : (gv == 2 ? ctcell_batch_kernel<T, false, true>(cpt) : ctcell_batch_kernel<T, false, false>(cpt));
}

template <typename T>
cudaError_t launch_mag_ctcell_batch(const MagArgs* args, const BlockMap* map, const PencilLaunch& L) {
    return launch_pencil_batch(ctcell_batch_kernel<T>(L.cpt, ghost_variant(L.fade, L.cg)), args, map, L);
}

template <typename T>
void (*fluid_kernel(int cpt, bool mhd, int gv))(const FluidArgs) {
    if (mhd)
        return gv == 1 ? fluid_kernel<T, true, true, false>(cpt)
                       : (gv == 2 ? fluid_kernel<T, true, false, true>(cpt) : fluid_kernel<T, true, false, false>(cpt));
    return gv == 1 ? fluid_kernel<T, false, true, false>(cpt)
                   : (gv == 2 ? fluid_kernel<T, false, false, true>(cpt) : fluid_kernel<T, false, false, false>(cpt));
}

template <typename T>
cudaError_t launch_fluid_sweep(const FluidArgs& a, const PencilLaunch& L, bool mhd) {
    return launch_pencil(fluid_kernel<T>(L.cpt, mhd, ghost_variant(L.fade, L.cg)), a, L);
}

template <typename T>
cudaError_t launch_mag_chain(const MagArgs& a, const PencilLaunch& L) {
    return launch_pencil(chain_kernel<T>(L.cpt, L.nqc, ghost_variant(L.fade, L.cg)), a, L);
}

template <typename T>
cudaError_t launch_mag_ctcell(const MagArgs& a, const PencilLaunch& L) {
    return launch_pencil(ctcell_kernel<T>(L.cpt, ghost_variant(L.fade, L.cg)), a, L);
}

// Allow a kernel the device's whole opt-in shared memory per block (minus its static shared
// memory).  The attribute belongs to the kernel, not to a launch, so it is raised to the maximum
// once instead of to one context's need (a smaller later value would break earlier contexts).
template <typename K>
cudaError_t allow_max_smem(K kern, int optin) {
    cudaFuncAttributes fa{};
    cudaError_t e = cudaFuncGetAttributes(&fa, kern);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}

template <typename T>
cudaError_t fluid_attributes(int cpt, int optin) {
    for (int v = 0; v < 6; ++v) {
        cudaError_t e = allow_max_smem(fluid_kernel<T>(cpt, v & 1, v >> 1), optin);
        if (e == cudaSuccess) e = allow_max_smem(fluid_batch_kernel<T>(cpt, v & 1, v >> 1), optin);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <typename T>
cudaError_t chain_attributes(int cpt, int optin) {
    for (int gv = 0; gv < 3; ++gv) {
        for (int nqc = 1; nqc <= (cpt <= 2 ? 2 : 1); ++nqc) {
            cudaError_t e = allow_max_smem(chain_kernel<T>(cpt, nqc, gv), optin);
            if (e == cudaSuccess) e = allow_max_smem(chain_batch_kernel<T>(cpt, nqc, gv), optin);
            if (e != cudaSuccess) return e;
        }
        cudaError_t e = allow_max_smem(ctcell_kernel<T>(cpt, gv), optin);
        if (e == cudaSuccess) e = allow_max_smem(ctcell_batch_kernel<T>(cpt, gv), optin);
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
    return cudaOccupancyMaxActiveClusters(n, fluid_kernel<T>(L.cpt, true, ghost_variant(L.fade, L.cg)), &lc);
}

}  // namespace img
