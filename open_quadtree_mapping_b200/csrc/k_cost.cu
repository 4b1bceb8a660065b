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

// floor(c + 0.5) for -0.5 <= c < 2^22 - 0.5, which equals the reference's
// (int)((double)c + 0.5) there, as HALF the integer n = floor(2c + 1): the
// sum c + (2^22 + 0.5) lies in [2^22, 2^23), where floats are spaced 0.5
// apart, so rounding it down gives 2^22 + n/2 exactly, and the bit pattern of
// that float minus the one of 2^22 is n.  The caller shifts right by one.
// The returned value is the bit pattern itself; kHalfBias = bits(2^22) / 2 is
// subtracted (folded into the image offset) after the shift.
__device__ __forceinline__ unsigned twice_round_bits(float c)
{
  return (unsigned)__float_as_int(__fadd_rd(c, 4194304.5f));
}
constexpr unsigned kHalfBias = 0x4A800000u >> 1;

// The 3x3 patch coordinates along one axis.  The reference computes
// (u + a*i) + b*j for i, j in {-1, 0, 1} (i the patch column, j the row).
// The products are exact (a*(+-1) = +-a, a*0 = +-0, and c +- 0 = c), so in
// both arithmetic modes the nine values are these correctly rounded sums:
// three column bases, then three rows each.  c[3*(j+1) + (i+1)].
__device__ __forceinline__ void patch_axis(float u, float a, float b, float (&c)[9])
{
  const float r[3] = {__fadd_rn(u, -a), u, __fadd_rn(u, a)};
#pragma unroll
  for (int i = 0; i < 3; ++i)
  {
    c[i] = __fadd_rn(r[i], -b);
    c[3 + i] = r[i];
    c[6 + i] = __fadd_rn(r[i], b);
  }
}

template <class A>
__global__ void __launch_bounds__(kFlatThreads)
    k_cost(const __grid_constant__ Batch B)
{
  __shared__ float4 s_pose[kMaxSlots * 3];
  __shared__ const uint8_t *s_img[kMaxSlots];
  __shared__ int s_w[kMaxSlots];
  int lb;
  const JobDesc &J = job_of(B, lb);
  const int D = J.D;
  const int F = J.F;
  // the job's (deduplicated) slots, staged once per block; every block
  // belongs to one job
  for (int i = threadIdx.x; i < F * 12; i += blockDim.x)
    reinterpret_cast<float *>(s_pose)[i] = slot_pose(B, J.slot_base + i / 12)[i % 12];
  for (int i = threadIdx.x; i < F; i += blockDim.x)
  {
    s_img[i] = slot_image(B, J.slot_base + i);
    s_w[i] = slot_weight(B, J.slot_base + i);
  }
  __syncthreads();
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
  // (int)(u + 0.5) in [2, W-2) exactly when u in [1.5, W-2.5) (both bounds
  // are floats, the comparisons exact; NaN fails)
  const float ulo = 1.5f, uhi = (float)W - 2.5f, vhi = (float)H - 2.5f;
  const unsigned bias = 0u - kHalfBias * ((unsigned)pitch + 1u);
  int sad = 0, nvalid = 0;
  for (int f = 0; f < F; ++f)
  {
    float T[12];
    const float4 t0 = s_pose[3 * f], t1 = s_pose[3 * f + 1], t2 = s_pose[3 * f + 2];
    T[0] = t0.x, T[1] = t0.y, T[2] = t0.z, T[3] = t0.w;
    T[4] = t1.x, T[5] = t1.y, T[6] = t1.z, T[7] = t1.w;
    T[8] = t2.x, T[9] = t2.y, T[10] = t2.z, T[11] = t2.w;
    const float3 q = A::apply(T, p);
    const float2 uv = A::project(q, cam);
    if (uv.x >= ulo && uv.x < uhi && uv.y >= ulo && uv.y < vhi)
    {
      const uint8_t *m = s_img[f];
      // The slot poses are validated as rigid on the host (|r00|+|r01| and
      // |r10|+|r11| <= 1.5), so every patch coordinate + 0.5 lies in
      // [0.5, W-0.5) x [0.5, H-0.5): no clamp needed.
      float px[9], py[9];
      patch_axis(uv.x, T[0], T[1], px);
      patch_axis(uv.y, T[4], T[5], py);
      unsigned s = 0;
#pragma unroll
      for (int k = 0; k < 9; ++k)
      {
        // offset = floor(py+0.5)*pitch + floor(px+0.5), in 32-bit wrap-around
        // arithmetic (the true offset is below 2^31)
        const unsigned hx = twice_round_bits(px[k]) >> 1;
        const unsigned hy = twice_round_bits(py[k]) >> 1;
        const unsigned off = hy * (unsigned)pitch + hx + bias;
        s = __usad((unsigned)patch[k % 3][k / 3], (unsigned)__ldg(m + off), s);
      }
      const int wgt = s_w[f];
      sad += wgt * (int)s;
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
