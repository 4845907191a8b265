// Launch entry points of the pencil kernels, compiled in their own translation units (one per
// kernel family and precision, built in parallel) and called by the host code.
#pragma once

#include "magnet_sweep.cuh"
#include "seg_fluid.cuh"
#include "seg_magnet.cuh"

namespace img {

// Launch shape of one pencil-kernel launch.
struct PencilLaunch {
    unsigned grid_x, grid_y;   // CTAs (grid_x = bundles x cluster size)
    unsigned block;            // threads per CTA
    size_t smem;               // dynamic shared memory per CTA
    int cluster;               // CTAs per cluster along the pencil
    int cpt;                   // cells per thread (1, 2 or 4)
    int nqc;                   // magnet chain: transverse components per CTA (1, or 2 with cpt <= 2)
    bool fade;                 // a fade BC on this sweep direction
    bool cg;                   // copy ghosts (single-CTA pencils, circ/const/fade shifts)
    bool init;                 // fluid sweep / chain: captures stored edges (overrides cg)
    int seg;                   // cells per thread of the segment fluid kernel (seg_fluid.cuh) or of the window
                               // magnet kernels (seg_magnet.cuh); 0: the pencil-tile kernels
    bool clu;                  // segment fluid kernel: one pencil along x per cluster (or per CTA with a
                               // ragged last segment), seg_fluid.cuh's CLU form
    cudaStream_t stream;
};

template <typename T> cudaError_t launch_fluid_sweep(const FluidArgs& a, const PencilLaunch& L, bool mhd);
template <typename T> cudaError_t launch_mag_chain(const MagArgs& a, const PencilLaunch& L);
template <typename T> cudaError_t launch_mag_ctcell(const MagArgs& a, const PencilLaunch& L);
// Batched forms: one launch over the CTAs of many grids; `args` and `map` are device arrays (one
// argument block per member, one BlockMap per CTA of the launch, L.grid_x CTAs).
template <typename T>
cudaError_t launch_fluid_sweep_batch(const FluidArgs* args, const BlockMap* map, const PencilLaunch& L, bool mhd);
// The batched fluid sweep over pencils that span a thread-block cluster (L.cluster > 1), defined in
// fluid_cluster.cu: that translation unit is compiled at ptxas -O1 (see there), and its kernels need
// their own shared-memory attributes (fluid_cluster_attributes).
template <typename T>
cudaError_t launch_fluid_sweep_batch_cluster(const FluidArgs* args, const BlockMap* map, const PencilLaunch& L, bool mhd);
template <typename T> cudaError_t fluid_cluster_attributes(int cpt, int optin);
template <typename T> cudaError_t launch_mag_chain_batch(const MagArgs* args, const BlockMap* map, const PencilLaunch& L);
template <typename T>
cudaError_t launch_mag_ctcell_batch(const MagArgs* args, const BlockMap* map, const PencilLaunch& L);
// Let every fluid (resp. chain and CT) kernel variant with `cpt` cells per thread, single and
// batched, use up to `optin` bytes of shared memory per block (the device's opt-in maximum).
template <typename T> cudaError_t fluid_attributes(int cpt, int optin);
template <typename T> cudaError_t chain_attributes(int cpt, int optin);
// Clusters of the MHD fluid kernel that can be co-resident for launch shape L (0: not schedulable).
template <typename T> cudaError_t fluid_max_clusters(const PencilLaunch& L, int* n);
// Shared-memory attributes of the segment fluid kernels (2, 3, 4 and 8 cells per thread; 2, 3 and 4 in
// FP64; the cluster forms with 2, 4 and 8, and 2 and 4).
template <typename T> cudaError_t fluid_seg_attributes(int optin);

}  // namespace img
