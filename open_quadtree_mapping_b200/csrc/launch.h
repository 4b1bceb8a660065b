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
// warps per block of the warp-per-cell kernels (BP sweep, extraction): the
// default and the largest the kernels are compiled for (the autotuner picks
// among 4, 8 and 16)
constexpr int kCellWarps = 8;
constexpr int kMaxCellWarps = 16;
// line solvers: one warp per line; rows per block of the row pass and
// columns per block (stripe width) of the column pass: defaults and maxima
constexpr int kRowWarps = 2;
constexpr int kColLines = 4;
constexpr int kMaxRowWarps = 4;
constexpr int kMaxColLines = 8;
// cost kernel: resident blocks of 256 threads per SM it is compiled for
constexpr int kCostBlocks = 5;
// longest lines the solvers' shared memory holds
constexpr int kMaxRowLen = 4096;
constexpr int kMaxColLen = 2048;
size_t row_solve_smem(int max_w, int rows = kRowWarps);
size_t col_solve_smem(int max_h, int lines = kColLines);

// shared memory one block may take
constexpr int kMaxBlockSmem = 227 * 1024;

// Launch shapes of one active job set (chosen by the engine's autotuner).
struct Tune
{
  int sweep_warps = kCellWarps;   // warps per block of the BP half-sweeps
  int extract_warps = kCellWarps; // warps per block of the extraction
  int row_warps = kRowWarps;      // rows per block of the row solve
  int col_lines = kColLines;      // columns per block of the column solve
  int cost_blocks = kCostBlocks;  // resident cost-kernel blocks per SM (3, 4 or 5)
};
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
// max_d: largest hypothesis count of the batch (sizes the shared tile);
// blocks_per_sm: 3, 4 or 5, the instance's register budget
void launch_cost(const Batch &B, int blocks, int arith, int max_d, cudaStream_t s,
                 int blocks_per_sm = kCostBlocks);
void launch_pyramid(const Batch &B, int blocks, int level, cudaStream_t s);
// writes the inherited messages of level `level` that its sweeps will read
// (cells the quadtree test skips; all unswept cells when iters < 2)
void launch_msg_inherit(const Batch &B, int blocks, int level, int iters, int qt_max,
                        cudaStream_t s);
// half-sweep `it` (0-based) of level `level`; `warps` per block.  inherit:
// half-sweeps 0 and 1 also write the inherited messages of their colour's
// cells the quadtree test skips (instead of launch_msg_inherit; the level
// must have at least two half-sweeps)
void launch_bp_sweep(const Batch &B, int blocks, int d, int level, int it, KParams kp, int arith,
                     cudaStream_t s, int warps = kCellWarps, int inherit = 0);
// a half-sweep of colour `parity` that reads every incoming message from the
// level's own buffers (all cells' starting messages already written)
void launch_bp_sweep_own(const Batch &B, int blocks, int d, int level, int parity, KParams kp,
                         int arith, cudaStream_t s, int warps = kCellWarps);
// Coarse BP levels in one launch (k_bp_coarse): levels hi down to lo, every
// one with at least two half-sweeps (their first two write the inherited
// messages), one cluster of kCoarseCtas blocks of kCoarseThreads threads per
// job, jobs j0 .. j0 + jobs - 1 of the batch (B.jobs null: the inline job).
constexpr int kCoarseCtas = 8;
constexpr int kCoarseThreads = 512;
struct CoarsePlan
{
  int lo, hi;
  int iters[kMaxLevels];
};
void launch_bp_coarse(const Batch &B, int j0, int jobs, int d, const CoarsePlan &plan,
                      KParams kp, int arith, cudaStream_t s);
void launch_extract(const Batch &B, int blocks, int d, int arith, cudaStream_t s,
                    int warps = kCellWarps);
void launch_row_solve(const Batch &B, int blocks, KParams kp, int arith, int max_w,
                      cudaStream_t s, int rows = kRowWarps);
void launch_col_solve(const Batch &B, int blocks, KParams kp, int arith, int max_h,
                      cudaStream_t s, int lines = kColLines);
// pixels per thread of the fusion transform and update (their blocks cover
// kFlatThreads times as many; the update walks its pixels as a pipeline)
constexpr int kFuseTransformPx = 4;
constexpr int kFuseUpdatePx = 8;
void launch_fuse_transform(const Batch &B, int blocks, int arith, cudaStream_t s);
// hole filling + posterior update (reads the z-buffer keys, leaves them set:
// the next frame's row solve resets them)
void launch_fuse_update(const Batch &B, int blocks, cudaStream_t s);
// out[i] = seeds[i].w (the fused variance sigma^2), n pixels
void launch_seed_variance(const float4 *seeds, float *out, long n, cudaStream_t s);

// Point cloud of one depth map (k_points.cu): out receives (x, y, z,
// intensity) per kept pixel in row-major order, *count (device) their number;
// ws holds point_cloud_workspace(W, H) bytes.
int point_cloud_tiles(int W, int H);
size_t point_cloud_workspace(int W, int H);
void launch_point_cloud(const float *depth, size_t stride, const uint8_t *ref, size_t pitch, int W,
                        int H, const Cam &cam, const float *T_world_ref, float4 *out, int *count,
                        void *ws, cudaStream_t s);

// ---------------------------------------------------------------------------
// Differentiable path (k_diff.cu).

// One BP level of one keyframe for the soft readout and the BP adjoint, with
// messages, adjoints and data terms of real type R: float for the
// differentiable product path, double for the gradient-check mode.
template <class R>
struct DiffBpR
{
  int W, H, D;           // image and hypotheses
  int w, h;              // cells of this level
  int level, parity, qt_max;
  const uint8_t *levels; // quadtree level map
  const R *data;         // data term of this level
  const R *S[4];         // messages read (a state snapshot, or the finals)
  R *A[4];               // adjoint of the messages, by direction
  float P1, P2;
  double *gP;            // dL/dP1, dL/dP2 (accumulated)
  float tau;             // readout temperature
  double step, min_inv;  // hypothesis depths
  float *sparse;         // readout output (W x H)
  const float *g_sparse; // its adjoint
};
using DiffBp = DiffBpR<float>;
using DiffBp64 = DiffBpR<double>;
template <class R>
struct MsgPtrsR
{
  R *m[4];
};
using MsgPtrs = MsgPtrsR<float>;
using MsgPtrs64 = MsgPtrsR<double>;
// soft readout at level-0 node cells: forward writes sparse; backward adds
// the belief adjoint to A (the four incoming messages of every node cell)
void launch_soft_readout(const DiffBp &a, int backward, cudaStream_t s);
void launch_soft_readout(const DiffBp64 &a, int backward, cudaStream_t s);
// adjoint of one half-sweep of colour a.parity: reads A at the updated cells
// (then zeroes it) and adds to A at the messages they read (a.S is the state
// the forward half-sweep read)
void launch_bp_sweep_bwd(const DiffBp &a, cudaStream_t s);
void launch_bp_sweep_bwd(const DiffBp64 &a, cudaStream_t s);
// parent.m[k] += sum of the (up to four) children's child.m[k], k = 0..3
void launch_msg_downsample_add(const MsgPtrs &child, int cw, int ch, const MsgPtrs &parent,
                               int pw, int ph, int D, cudaStream_t s);
void launch_msg_downsample_add(const MsgPtrs64 &child, int cw, int ch, const MsgPtrs64 &parent,
                               int pw, int ph, int D, cudaStream_t s);
// FP64 BP forward of the gradient-check mode (the product's BP is FP32):
// out[i] = in[i] widened; the pyramid of data terms (children summed x
// offset outer, y offset inner); every cell of a level starting from its
// parent's messages (zeros when parent is null), as the reference's
// copy-down; one half-sweep of colour a.parity updating M in place (a.S
// unused)
void launch_widen(const float *in, double *out, long n, cudaStream_t s);
void launch_pyramid64(const double *fine, int fw, int fh, double *coarse, int cw, int ch, int D,
                      cudaStream_t s);
void launch_msg_inherit_all64(const MsgPtrs64 *parent, int pw, const MsgPtrs64 &child, int cw,
                              int ch, int D, cudaStream_t s);
void launch_bp_sweep_fwd64(const DiffBp64 &a, const MsgPtrs64 &M, cudaStream_t s);

// Weighted upsampling of one image (FP64 line solves).
struct DiffUp
{
  int W, H;
  const uint8_t *img;
  size_t pitch;
  const float *omega;     // W x H edge-weight factors
  double lam, sigma, row_closing, col_closing;
  const float *sparse;    // input
  float *dense;           // output
  double *sd, *si;        // row-pass results (depth, indicator)
  double *td, *ti;        // column-pass results
  double *cp;             // Thomas scratch
  double *ud, *ui;        // adjoint scratch
  const float *g_dense;   // incoming adjoint
  float *g_sparse, *g_omega;
};
void launch_upw_forward(const DiffUp &u, cudaStream_t s);
void launch_upw_backward(const DiffUp &u, cudaStream_t s);

struct DiffFuse
{
  int W, H;
  const float *depth_in;  // upsampled depth before fusion
  const float4 *seeds_in; // the transformed previous seeds
  const int32_t *table;   // source seed per pixel (0 = none)
  const float *g_fused;
  float *g_depth;
};
void launch_fuse_bwd(const DiffFuse &f, cudaStream_t s);

// supported hypothesis-count classes of the BP kernels
bool bp_supported_d(int d);
// cells one warp of the BP sweep / extraction handles for d hypotheses
int bp_cells_per_warp(int d);

} // namespace qm
