// Host-side launchers of the pipeline kernels (one launch per stage over all
// jobs of a batch).  `prefix` is the device copy of the per-job block prefix
// of that stage and `blocks` its last entry.
#pragma once

#include <cuda_runtime.h>

#include "qm_internal.cuh"

namespace qm
{

// threads per block of the flat per-element kernels
constexpr int kFlatThreads = 256;
// warps per block of the warp-per-cell kernels (BP sweep, extraction)
constexpr int kCellWarps = 8;
// line solvers: one warp per line; rows per block of the row pass and
// columns per block (stripe width) of the column pass
constexpr int kRowWarps = 2;
constexpr int kColLines = 4;
// longest lines the solvers' shared memory holds
constexpr int kMaxRowLen = 4096;
constexpr int kMaxColLen = 2048;
size_t row_solve_smem(int max_w);
size_t col_solve_smem(int max_h);
void prepare_upsample_kernels();

// blocks of the quadtree launch for one W x H image
int quadtree_blocks(int W, int H, int qt_max);

// Every launcher takes the batch by value (the kernels receive it as a
// __grid_constant__ parameter); B.prefix must point at the stage's prefix.
void launch_quadtree(const Batch &B, int blocks, KParams kp, cudaStream_t s);
// cells per block of the cost kernel (one tile of a cell row)
constexpr int kCostCells = 32;
constexpr int kMaxHyp = 128;
int cost_blocks(int cw, int ch);
// max_d: largest hypothesis count of the batch (sizes the shared tile)
void launch_cost(const Batch &B, int blocks, int arith, int max_d, cudaStream_t s);
void launch_pyramid(const Batch &B, int blocks, int level, cudaStream_t s);
// writes the inherited messages of level `level` that its sweeps will read
// (cells the quadtree test skips; all unswept cells when iters < 2)
void launch_msg_inherit(const Batch &B, int blocks, int level, int iters, int qt_max,
                        cudaStream_t s);
// half-sweep `it` (0-based) of level `level`
void launch_bp_sweep(const Batch &B, int blocks, int d, int level, int it, KParams kp, int arith,
                     cudaStream_t s);
void launch_extract(const Batch &B, int blocks, int d, int arith, cudaStream_t s);
void launch_row_solve(const Batch &B, int blocks, KParams kp, int arith, int max_w,
                      cudaStream_t s);
void launch_col_solve(const Batch &B, int blocks, KParams kp, int arith, int max_h,
                      cudaStream_t s);
void launch_fuse_transform(const Batch &B, int blocks, int arith, cudaStream_t s);
void launch_fuse_fill(const Batch &B, int blocks, cudaStream_t s);
void launch_fuse_update(const Batch &B, int blocks, cudaStream_t s);
// out[i] = seeds[i].w (the fused variance sigma^2), n pixels
void launch_seed_variance(const float4 *seeds, float *out, long n, cudaStream_t s);

// supported hypothesis-count classes of the BP kernels
bool bp_supported_d(int d);
// cells one warp of the BP sweep / extraction handles for d hypotheses
int bp_cells_per_warp(int d);

} // namespace qm
