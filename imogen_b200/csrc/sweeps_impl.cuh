// Definitions of the launch entry points declared in sweeps.cuh.  Each translation unit that
// includes this file instantiates them for one precision.
#pragma once

#include "sweeps.cuh"

namespace img {

// Launch configuration of a pencil kernel: the cluster shape, and for single-CTA pencils programmatic
// stream serialization (the kernel may be scheduled while the previous kernel of the stream runs its
// last stage; the kernel bodies wait for it with pdl_wait before reading anything it wrote).
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
    if (L.cluster == 1) {
        attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[1].val.programmaticStreamSerializationAllowed = 1;
        lc.numAttrs = 2;
    }
    return lc;
}

template <typename Args>
cudaError_t launch_pencil_batch(void (*kern)(const Args*, const BlockMap*), const Args* args, const BlockMap* map,
                                const PencilLaunch& L) {
    cudaLaunchAttribute attr[2];
    cudaLaunchConfig_t lc = pencil_config(L, attr);
    return cudaLaunchKernelEx(&lc, kern, args, map);
}

template <typename Args>
cudaError_t launch_pencil(void (*kern)(const Args), const Args& a, const PencilLaunch& L) {
    cudaLaunchAttribute attr[2];
    cudaLaunchConfig_t lc = pencil_config(L, attr);
    return cudaLaunchKernelEx(&lc, kern, a);
}

// Kernel variant of a pencil launch (see kv_fade/kv_cg/kv_init): halo jobs (0), with fade (1), copy
// ghosts (2), the stored-edge capturing forms of 0 and 1 (3, 4), which first sweeps use, and copy
// ghosts with fade (5).
inline int kernel_variant(bool fade, bool cg, bool init) {
    if (init) return fade ? 4 : 3;
    if (cg) return fade ? 5 : 2;
    return fade ? 1 : 0;
}

template <typename T, bool MHD, int V>
void (*fluid_kernel_v(int cpt))(const FluidArgs) {
    switch (cpt) {
        case 1: return fluid_sweep_kernel<T, MHD, 1, V>;
        case 2: return fluid_sweep_kernel<T, MHD, 2, V>;
        default: return fluid_sweep_kernel<T, MHD, 4, V>;
    }
}

template <typename T, bool MHD, int V>
void (*fluid_batch_kernel_v(int cpt))(const FluidArgs*, const BlockMap*) {
    switch (cpt) {
        case 1: return fluid_sweep_batch_kernel<T, MHD, 1, V>;
        case 2: return fluid_sweep_batch_kernel<T, MHD, 2, V>;
        default: return fluid_sweep_batch_kernel<T, MHD, 4, V>;
    }
}

template <typename T, int V>
void (*chain_kernel_v(int cpt, int nqc))(const MagArgs) {
    if (nqc == 2) return cpt == 1 ? mag_chain_kernel<T, 1, 2, V> : mag_chain_kernel<T, 2, 2, V>;
    switch (cpt) {
        case 1: return mag_chain_kernel<T, 1, 1, V>;
        case 2: return mag_chain_kernel<T, 2, 1, V>;
        default: return mag_chain_kernel<T, 4, 1, V>;
    }
}

template <typename T, int V>
void (*chain_batch_kernel_v(int cpt, int nqc))(const MagArgs*, const BlockMap*) {
    if (nqc == 2) return cpt == 1 ? mag_chain_batch_kernel<T, 1, 2, V> : mag_chain_batch_kernel<T, 2, 2, V>;
    switch (cpt) {
        case 1: return mag_chain_batch_kernel<T, 1, 1, V>;
        case 2: return mag_chain_batch_kernel<T, 2, 1, V>;
        default: return mag_chain_batch_kernel<T, 4, 1, V>;
    }
}

template <typename T, bool MHD>
void (*fluid_kernel_m(int cpt, int v))(const FluidArgs) {
    switch (v) {
        case 1: return fluid_kernel_v<T, MHD, 1>(cpt);
        case 2: return fluid_kernel_v<T, MHD, 2>(cpt);
        case 3: return fluid_kernel_v<T, MHD, 3>(cpt);
        case 4: return fluid_kernel_v<T, MHD, 4>(cpt);
        case 5: return fluid_kernel_v<T, MHD, 5>(cpt);
        default: return fluid_kernel_v<T, MHD, 0>(cpt);
    }
}

template <typename T, bool MHD>
void (*fluid_batch_kernel_m(int cpt, int v))(const FluidArgs*, const BlockMap*) {
    switch (v) {
        case 1: return fluid_batch_kernel_v<T, MHD, 1>(cpt);
        case 2: return fluid_batch_kernel_v<T, MHD, 2>(cpt);
        case 3: return fluid_batch_kernel_v<T, MHD, 3>(cpt);
        case 4: return fluid_batch_kernel_v<T, MHD, 4>(cpt);
        case 5: return fluid_batch_kernel_v<T, MHD, 5>(cpt);
        default: return fluid_batch_kernel_v<T, MHD, 0>(cpt);
    }
}

template <typename T>
void (*fluid_kernel(int cpt, bool mhd, int v))(const FluidArgs) {
    return mhd ? fluid_kernel_m<T, true>(cpt, v) : fluid_kernel_m<T, false>(cpt, v);
}

template <typename T>
void (*fluid_batch_kernel(int cpt, bool mhd, int v))(const FluidArgs*, const BlockMap*) {
    return mhd ? fluid_batch_kernel_m<T, true>(cpt, v) : fluid_batch_kernel_m<T, false>(cpt, v);
}

template <typename T>
void (*chain_kernel(int cpt, int nqc, int v))(const MagArgs) {
    switch (v) {
        case 1: return chain_kernel_v<T, 1>(cpt, nqc);
        case 2: return chain_kernel_v<T, 2>(cpt, nqc);
        case 3: return chain_kernel_v<T, 3>(cpt, nqc);
        case 4: return chain_kernel_v<T, 4>(cpt, nqc);
        case 5: return chain_kernel_v<T, 5>(cpt, nqc);
        default: return chain_kernel_v<T, 0>(cpt, nqc);
    }
}

template <typename T>
void (*chain_batch_kernel(int cpt, int nqc, int v))(const MagArgs*, const BlockMap*) {
    switch (v) {
        case 1: return chain_batch_kernel_v<T, 1>(cpt, nqc);
        case 2: return chain_batch_kernel_v<T, 2>(cpt, nqc);
        case 3: return chain_batch_kernel_v<T, 3>(cpt, nqc);
        case 4: return chain_batch_kernel_v<T, 4>(cpt, nqc);
        case 5: return chain_batch_kernel_v<T, 5>(cpt, nqc);
        default: return chain_batch_kernel_v<T, 0>(cpt, nqc);
    }
}

// The CT kernel captures no stored edges: its variant ignores `init` (0 jobs, 1 fade, 2 cg, 3 both).
inline int ct_variant(bool fade, bool cg) { return (fade ? 1 : 0) | (cg ? 2 : 0); }

// Segment fluid kernels by cells per thread (2, 3, 4 and 8; FP64: 2, 3 and 4).  3 serves pencils of
// 3 cells held whole by one thread.
template <typename T, bool MHD>
void (*fluid_seg_kernel_c(int C))(const FluidArgs) {
    if constexpr (sizeof(T) == 4) {
        if (C == 8) return fluid_seg_kernel<T, MHD, 8>;
    }
    if (C == 3) return fluid_seg_kernel<T, MHD, 3>;
    return C == 2 ? fluid_seg_kernel<T, MHD, 2> : fluid_seg_kernel<T, MHD, 4>;
}

template <typename T, bool MHD>
void (*fluid_seg_batch_kernel_c(int C))(const FluidArgs*, const BlockMap*) {
    if constexpr (sizeof(T) == 4) {
        if (C == 8) return fluid_seg_batch_kernel<T, MHD, 8>;
    }
    if (C == 3) return fluid_seg_batch_kernel<T, MHD, 3>;
    return C == 2 ? fluid_seg_batch_kernel<T, MHD, 2> : fluid_seg_batch_kernel<T, MHD, 4>;
}

// With artificial viscosity: 2 and 4 cells per thread.
template <typename T, bool MHD, int VT>
void (*fluid_seg_visc_kernel_c(int C))(const FluidArgs) {
    return C == 2 ? fluid_seg_kernel<T, MHD, 2, VT> : fluid_seg_kernel<T, MHD, 4, VT>;
}

template <typename T>
void (*fluid_seg_kernel_p(int C, bool mhd, int visc = VISC_NONE))(const FluidArgs) {
    if (visc == VISC_NR) return mhd ? fluid_seg_visc_kernel_c<T, true, VISC_NR>(C) : fluid_seg_visc_kernel_c<T, false, VISC_NR>(C);
    if (visc == VISC_CSW) return mhd ? fluid_seg_visc_kernel_c<T, true, VISC_CSW>(C) : fluid_seg_visc_kernel_c<T, false, VISC_CSW>(C);
    return mhd ? fluid_seg_kernel_c<T, true>(C) : fluid_seg_kernel_c<T, false>(C);
}

template <typename T>
void (*fluid_seg_batch_kernel_p(int C, bool mhd))(const FluidArgs*, const BlockMap*) {
    return mhd ? fluid_seg_batch_kernel_c<T, true>(C) : fluid_seg_batch_kernel_c<T, false>(C);
}

// Cluster (CLU) forms of the segment fluid kernel: 2, 4 and 8 cells per thread (FP64: 2 and 4).
template <typename T, bool MHD>
void (*fluid_seg_clu_kernel_c(int C))(const FluidArgs) {
    if constexpr (sizeof(T) == 4) {
        if (C == 8) return fluid_seg_clu_kernel<T, MHD, 8>;
    }
    return C == 2 ? fluid_seg_clu_kernel<T, MHD, 2> : fluid_seg_clu_kernel<T, MHD, 4>;
}

template <typename T, bool MHD>
void (*fluid_seg_clu_batch_kernel_c(int C))(const FluidArgs*, const BlockMap*) {
    if constexpr (sizeof(T) == 4) {
        if (C == 8) return fluid_seg_clu_batch_kernel<T, MHD, 8>;
    }
    return C == 2 ? fluid_seg_clu_batch_kernel<T, MHD, 2> : fluid_seg_clu_batch_kernel<T, MHD, 4>;
}

template <typename T>
void (*fluid_seg_clu_kernel_p(int C, bool mhd))(const FluidArgs) {
    return mhd ? fluid_seg_clu_kernel_c<T, true>(C) : fluid_seg_clu_kernel_c<T, false>(C);
}

template <typename T>
void (*fluid_seg_clu_batch_kernel_p(int C, bool mhd))(const FluidArgs*, const BlockMap*) {
    return mhd ? fluid_seg_clu_batch_kernel_c<T, true>(C) : fluid_seg_clu_batch_kernel_c<T, false>(C);
}

template <typename T>
cudaError_t launch_fluid_sweep_batch(const FluidArgs* args, const BlockMap* map, const PencilLaunch& L, bool mhd) {
    if (L.seg && L.clu) return launch_pencil_batch(fluid_seg_clu_batch_kernel_p<T>(L.seg, mhd), args, map, L);
    if (L.seg) return launch_pencil_batch(fluid_seg_batch_kernel_p<T>(L.seg, mhd), args, map, L);
    if (L.cluster > 1) return launch_fluid_sweep_batch_cluster<T>(args, map, L, mhd);
    return launch_pencil_batch(fluid_batch_kernel<T>(L.cpt, mhd, kernel_variant(L.fade, L.cg, L.init)), args, map, L);
}

// Window magnet kernels by cells per thread (2, 3, 4, 8).
template <typename T>
void (*chain_win_kernel(int C))(const MagArgs) {
    if (C == 3) return mag_chain_win_kernel<T, 3>;
    return C == 2 ? mag_chain_win_kernel<T, 2> : (C == 8 ? mag_chain_win_kernel<T, 8> : mag_chain_win_kernel<T, 4>);
}
template <typename T>
void (*ct_win_kernel(int C))(const MagArgs) {
    if (C == 3) return mag_ct_win_kernel<T, 3>;
    return C == 2 ? mag_ct_win_kernel<T, 2> : (C == 8 ? mag_ct_win_kernel<T, 8> : mag_ct_win_kernel<T, 4>);
}
template <typename T>
void (*chain_win_batch_kernel(int C))(const MagArgs*, const BlockMap*) {
    if (C == 3) return mag_chain_win_batch_kernel<T, 3>;
    return C == 2 ? mag_chain_win_batch_kernel<T, 2> : (C == 8 ? mag_chain_win_batch_kernel<T, 8> : mag_chain_win_batch_kernel<T, 4>);
}
template <typename T>
void (*ct_win_batch_kernel(int C))(const MagArgs*, const BlockMap*) {
    if (C == 3) return mag_ct_win_batch_kernel<T, 3>;
    return C == 2 ? mag_ct_win_batch_kernel<T, 2> : (C == 8 ? mag_ct_win_batch_kernel<T, 8> : mag_ct_win_batch_kernel<T, 4>);
}

template <typename T>
cudaError_t launch_mag_chain_batch(const MagArgs* args, const BlockMap* map, const PencilLaunch& L) {
    if (L.seg) return launch_pencil_batch(chain_win_batch_kernel<T>(L.seg), args, map, L);
    return launch_pencil_batch(chain_batch_kernel<T>(L.cpt, L.nqc, kernel_variant(L.fade, L.cg, L.init)), args, map, L);
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
    switch (gv) {
        case 1: return ctcell_kernel<T, true, false>(cpt);
        case 2: return ctcell_kernel<T, false, true>(cpt);
        case 3: return ctcell_kernel<T, true, true>(cpt);
        default: return ctcell_kernel<T, false, false>(cpt);
    }
}

template <typename T>
void (*ctcell_batch_kernel(int cpt, int gv))(const MagArgs*, const BlockMap*) {
    switch (gv) {
        case 1: return ctcell_batch_kernel<T, true, false>(cpt);
        case 2: return ctcell_batch_kernel<T, false, true>(cpt);
        case 3: return ctcell_batch_kernel<T, true, true>(cpt);
        default: return ctcell_batch_kernel<T, false, false>(cpt);
    }
}

template <typename T>
cudaError_t launch_mag_ctcell_batch(const MagArgs* args, const BlockMap* map, const PencilLaunch& L) {
    if (L.seg) return launch_pencil_batch(ct_win_batch_kernel<T>(L.seg), args, map, L);
    return launch_pencil_batch(ctcell_batch_kernel<T>(L.cpt, ct_variant(L.fade, L.cg)), args, map, L);
}

template <typename T>
cudaError_t launch_fluid_sweep(const FluidArgs& a, const PencilLaunch& L, bool mhd) {
    if (L.seg && L.clu) return launch_pencil(fluid_seg_clu_kernel_p<T>(L.seg, mhd), a, L);
    if (L.seg) return launch_pencil(fluid_seg_kernel_p<T>(L.seg, mhd, a.visc), a, L);
    return launch_pencil(fluid_kernel<T>(L.cpt, mhd, kernel_variant(L.fade, L.cg, L.init)), a, L);
}

template <typename T>
cudaError_t launch_mag_chain(const MagArgs& a, const PencilLaunch& L) {
    if (L.seg) return launch_pencil(chain_win_kernel<T>(L.seg), a, L);
    return launch_pencil(chain_kernel<T>(L.cpt, L.nqc, kernel_variant(L.fade, L.cg, L.init)), a, L);
}

template <typename T>
cudaError_t launch_mag_ctcell(const MagArgs& a, const PencilLaunch& L) {
    if (L.seg) return launch_pencil(ct_win_kernel<T>(L.seg), a, L);
    return launch_pencil(ctcell_kernel<T>(L.cpt, ct_variant(L.fade, L.cg)), a, L);
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
    for (int v = 0; v < 12; ++v) {
        cudaError_t e = allow_max_smem(fluid_kernel<T>(cpt, v & 1, v >> 1), optin);
        if (e == cudaSuccess) e = allow_max_smem(fluid_batch_kernel<T>(cpt, v & 1, v >> 1), optin);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <typename T>
cudaError_t fluid_seg_attributes(int optin) {
    for (int C : {2, 3, 4, 8}) {
        if (sizeof(T) == 8 && C == 8) continue;
        for (int mhd = 0; mhd < 2; ++mhd) {
            cudaError_t e = allow_max_smem(fluid_seg_kernel_p<T>(C, mhd != 0), optin);
            if (e == cudaSuccess) e = allow_max_smem(fluid_seg_batch_kernel_p<T>(C, mhd != 0), optin);
            for (int vt : {VISC_NR, VISC_CSW})
                if (e == cudaSuccess && (C == 2 || C == 4)) e = allow_max_smem(fluid_seg_kernel_p<T>(C, mhd != 0, vt), optin);
            if (e == cudaSuccess && C != 3) e = allow_max_smem(fluid_seg_clu_kernel_p<T>(C, mhd != 0), optin);
            if (e == cudaSuccess && C != 3) e = allow_max_smem(fluid_seg_clu_batch_kernel_p<T>(C, mhd != 0), optin);
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

template <typename T>
cudaError_t chain_attributes(int cpt, int optin) {
    for (int v = 0; v < 6; ++v) {
        for (int nqc = 1; nqc <= (cpt <= 2 ? 2 : 1); ++nqc) {
            cudaError_t e = allow_max_smem(chain_kernel<T>(cpt, nqc, v), optin);
            if (e == cudaSuccess) e = allow_max_smem(chain_batch_kernel<T>(cpt, nqc, v), optin);
            if (e != cudaSuccess) return e;
        }
    }
    for (int v = 0; v < 4; ++v) {
        cudaError_t e = allow_max_smem(ctcell_kernel<T>(cpt, v), optin);
        if (e == cudaSuccess) e = allow_max_smem(ctcell_batch_kernel<T>(cpt, v), optin);
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
    return cudaOccupancyMaxActiveClusters(n, fluid_kernel<T>(L.cpt, true, kernel_variant(L.fade, L.cg, L.init)), &lc);
}

}  // namespace img
