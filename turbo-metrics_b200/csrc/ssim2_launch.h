// ssim2_launch.h -- host-side entry points of the kernels in ssim2_kernels.cu.
#pragma once
#include <cuda_runtime.h>

#include "ssim2_device.cuh"

namespace s2 {
const double *host_weights();
cudaError_t upload_weights();
cudaError_t configure_kernels();
size_t fused_smem_bytes();
int fused_blocks_per_sm(int storage);
// prep over the pyramid blocks [first_block, end_block) (absolute numbering
// of blk_first), fused over the tiles [first_tile, end_tile) with its own
// zeroed work counter.  out: 1 XYB planes (SSIMULACRA2), 2 Lab planes
// (DSSIM), 3 both from one pass.  fmt: the input format shared by every
// pair of the launch (a kernel compiled for it), or -1 for a mix.
cudaError_t launch_pyramid(int storage, const DevPair *pairs, int npairs, const int *blk_first, int first_block,
                           int end_block, const ColorConsts &cc, const float *lut, int grid, cudaStream_t st,
                           int out = 1, int fmt = -1);
// The tile pass's bounded waits: err is a device word (zeroed before the
// submission) that a pass whose row copies time out sets (launch_finalize
// then marks every pair S2_ERR_TIMEOUT); wait_cycles bounds each wait (SM
// clock cycles); drop_item >= 0 withholds the row copies of that work item
// so that its waits run out (the failure test; -1 in normal use).
struct TileCheck {
    int *err;
    long long wait_cycles;
    int drop_item;
};
TileCheck tile_check(int *err);  // the process-wide setting (s2_debug_tile_timeout)
cudaError_t launch_fused(int storage, const DevPair *pairs, const Seg *segs, int nseg, int first_tile,
                         int end_tile, int *counter, const TileCheck &ck, double *partials, int grid,
                         cudaStream_t st);
cudaError_t launch_iir(int storage, const DevPair *pairs, const IirSeg *vsegs, int nvseg, int vtotal,
                       const IirSeg *hsegs, int nhseg, int htotal, double *partials, cudaStream_t st);
// Copy `bytes` (a multiple of 16, both pointers 16-byte aligned) from
// page-locked host memory, through its device mapping, with a kernel: no copy
// engine, so the copy is not queued behind other streams' large uploads.
cudaError_t launch_desc_copy(void *dst, const void *src_host_mapped, size_t bytes, cudaStream_t st);
// The fused pass over the tiles [first_tile, end_tile) of one scale of one
// pair, also storing each pixel's three error-map values to `maps` (9 float
// planes [channel][ssim, artifact, detail], mpitch floats per row, mplane
// floats per plane).
cudaError_t launch_fused_export(int storage, const DevPair *pairs, const Seg *segs, int nseg,
                                int first_tile, int end_tile, int *counter, const TileCheck &ck, double *partials,
                                float *maps,
                                long long mpitch, long long mplane, int grid, cudaStream_t st);
cudaError_t launch_finalize(const DevPair *pairs, int npairs, const double *partials, const int *err,
                            DevResult *out, cudaStream_t st);

// DSSIM over the Lab planes of a submission (dssim_kernels.cu): the clamp
// pass (levels clamped to 8 pixels, pairs with clamp_from < 5), the tile
// pass (SSIM map and per-tile sums), the per-level means, the per-tile
// |avg - ssim| sums and the per-pair result.  `partials` holds 2 * ntiles
// doubles, `avg` 5 floats per pair.  write_all: the submission scores DSSIM
// only, so the final kernel also fills the SSIMULACRA2 fields of the result.
cudaError_t configure_dssim_kernels();
cudaError_t launch_dssim(const DsPair *pairs, int npairs, const DsSeg *segs, int nseg, int ntiles, bool clamp,
                         double *partials, float *avg, DevResult *out, bool write_all, int num_sms,
                         cudaStream_t st);
}  // namespace s2
