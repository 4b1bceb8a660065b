// Multi-view matching cost at quadtree nodes (image_to_cost +
// normalize_the_cost, depth_extract.cu:135-244 of the reference).
//
// One thread per (cell, hypothesis); consecutive threads are consecutive
// hypotheses of a cell, so the cost row of a cell (the PIXEL_COST layout,
// hypotheses contiguous) is written coalesced.  Each thread loops over the
// measurement slots itself and accumulates the 3x3 SAD as an integer: every
// term is an integer intensity difference, so the sum is exact and equal to
// the reference's shared-memory tree over slots.  The projection follows the
// reference's arithmetic (ArithRef) or IEEE rounding (ArithIeee).
//
// Cells that are not node origins, or touch the border (x <= 0, y <= 0,
// x >= W-1, y >= H-1), get cost 0 for every hypothesis, as the reference's
// zeroed cost image does.  A node with no valid slot gets 100.  Every node
// cost is then divided by the cell's writer count, which in the reference is
// the number of hypotheses: each hypothesis thread of slot row 0 adds 1 to it
// (depth_extract.cu:219-228), and normalize_the_cost divides by it
// (depth_extract.cu:231-244).
//
// Bytes per cell: 9 reference pixels + D*F*9 measurement gathers (u8, mostly
// L1/L2 hits along the epipolar segment) + 4*D written.
#include "launch.h"

namespace qm
{

namespace
{

template <class A>
__global__ void __launch_bounds__(kFlatThreads)
    k_cost(const __grid_constant__ Batch B)
{
  int lb;
  const JobDesc &J = job_of(B, lb);
  const int D = J.D;
  const long t = (long)lb * blockDim.x + threadIdx.x;
  const int ncell = J.cw * J.ch;
  if (t >= (long)ncell * D)
    return;
  const int cell = (int)(t / D);
  const int d = (int)(t - (long)cell * D);
  const int cx = cell % J.cw, cy = cell / J.cw;
  const int x = cx * 4, y = cy * 4;
  const int W = J.W, H = J.H;
  float *out = J.lv[0].data + (size_t)cell * D + d;
  const int size = 1 << J.levels[(size_t)y * W + x];
  if (x >= W - 1 || y >= H - 1 || x <= 0 || y <= 0 || x % size != 0 || y % size != 0)
  {
    *out = 0.0f;
    return;
  }
  int patch[3][3];
  const uint8_t *r = J.ref + (size_t)(y - 1) * J.ref_pitch + (x - 1);
#pragma unroll
  for (int jj = 0; jj < 3; ++jj)
#pragma unroll
    for (int ii = 0; ii < 3; ++ii)
      patch[ii][jj] = __ldg(r + (size_t)jj * J.ref_pitch + ii);

  const Cam cam{J.fx, J.fy, J.cx, J.cy};
  const float3 dir = A::ray((float)x, (float)y, cam);
  const float depth = A::hyp_depth(J.step, J.min_inv, d);
  const float3 p = A::scale(dir, depth);
  const int pitch = J.slot_pitch;
  int sad = 0, nvalid = 0;
  for (int f = 0; f < J.F; ++f)
  {
    // generic loads: in single-keyframe calls the poses live in the kernel
    // parameter, not in global memory
    const float *Tg = slot_pose(B, J.slot_base + f);
    float T[12];
#pragma unroll
    for (int k = 0; k < 12; ++k)
      T[k] = Tg[k];
    const float3 q = A::apply(T, p);
    const float2 uv = A::project(q, cam);
    // (int)(u + 0.5) in double in the reference; round_px is its exact
    // single-precision equivalent for the ranges these tests accept
    const int px = round_px(uv.x);
    const int py = round_px(uv.y);
    if (px >= 2 && px < W - 2 && py >= 2 && py < H - 2)
    {
      const uint8_t *m = slot_image(B, J.slot_base + f);
      const float u2u = T[0], u2v = T[4], v2u = T[1], v2v = T[5];
      int s = 0;
#pragma unroll
      for (int jj = -1; jj <= 1; ++jj)
#pragma unroll
        for (int ii = -1; ii <= 1; ++ii)
        {
          // In range for any rotation (|r00| + |r01| <= sqrt(2)); the clamp
          // only guards against non-rigid poses.
          const int chx = min(max(round_px(A::patch_coord(uv.x, u2u, ii, v2u, jj)), 0), W - 1);
          const int chy = min(max(round_px(A::patch_coord(uv.y, u2v, ii, v2v, jj)), 0), H - 1);
          s += abs(patch[ii + 1][jj + 1] - (int)__ldg(m + (size_t)chy * pitch + chx));
        }
      const int wgt = slot_weight(B, J.slot_base + f);
      sad += wgt * s;
      nvalid += wgt;
    }
  }
  float c = nvalid > 0 ? A::sad_norm((float)sad, (float)nvalid) : 100.0f;
  const int add_num = D; // writer count of the cell (see above)
  *out = A::div(c, (float)add_num);
}

} // namespace

void launch_cost(const Batch &B, int blocks, int arith, cudaStream_t s)
{
  if (arith == QM_ARITH_IEEE)
    k_cost<ArithIeee><<<blocks, kFlatThreads, 0, s>>>(B);
  else
    k_cost<ArithRef><<<blocks, kFlatThreads, 0, s>>>(B);
}

} // namespace qm
