// Multi-view matching cost at quadtree nodes (image_to_cost +
// normalize_the_cost, depth_extract.cu:135-244 of the reference).
//
// A block owns a tile of kCostCells consecutive cells of one cell row.  Warp
// 0 finds the tile's node cells (ballot) and stages, per node, its ray and
// 3x3 reference patch in shared memory; the block also stages the slot poses
// and the hypothesis depths.  Thread t then owns node t % n (n nodes in the
// tile) and every (256 / n)-th hypothesis from t / n on, so the lanes of a
// warp evaluate neighbouring nodes at one depth: their projections are
// neighbours in the slot image and a gather touches few cache lines; the
// node's ray and patch stay in registers.  Each pair loops over the
// measurement slots and accumulates the 3x3 SAD as an integer: every term is
// an integer intensity difference, so the sum is exact and equal to the
// reference's shared-memory tree over slots.  The projection follows the
// reference's arithmetic (ArithRef) or IEEE rounding (ArithIeee).  The tile's
// costs are assembled in shared memory and written as one contiguous run.
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

// floor(c + 0.5) for -0.5 <= c < 2^23 - 0.5, which equals the reference's
// (int)((double)c + 0.5) there, in one rounded operation: 2^23 + 0.5 is not
// a float, but it is the exact product 24929 * 336.5 (24929 = 97 * 257,
// 336.5 = 673 / 2), so a fused multiply-add rounded down evaluates
// RD(2^23 + 0.5 + c) with a single rounding.  That sum lies in [2^23, 2^24),
// where floats are spaced 1 apart, so the result is 2^23 + floor(c + 0.5)
// exactly, and its bit pattern minus kBias = bits(2^23) is the integer.  The
// returned value is the bit pattern; kBias is subtracted (folded into the
// image offset) by the caller.
__device__ __forceinline__ unsigned round_bits(float c)
{
  return (unsigned)__float_as_int(__fmaf_rd(24929.0f, 336.5f, c));
}
constexpr unsigned kBias = 0x4B000000u;

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

// MINB resident blocks of 256 threads per SM (at most 48, 64 or 80
// registers for 5, 4 or 3): more resident warps against fewer spilled
// values.  The balance depends on the hypothesis and slot counts, so the
// engine's autotuner picks it per stream set (measured on a B200: 32 x
// 752x480 with 64 hypotheses and 5 slots 0.969 ms at 4 blocks against 1.022
// at 5; at 8 x 1920x1080 with 128 hypotheses and 20 slots the tuner also
// picks 4, 8.13 ms against 8.90 with 5).
template <class A, int MINB>
__global__ void __launch_bounds__(kFlatThreads, MINB)
    k_cost(const __grid_constant__ Batch B)
{
  // costs of the tile, [kCostCells][D + 1] (the padding keeps lanes that
  // store one hypothesis of different cells on different banks)
  extern __shared__ float s_out[];
  __shared__ float4 s_pose[kMaxSlots * 3];
  __shared__ const uint8_t *s_img[kMaxSlots];
  __shared__ int s_w[kMaxSlots];
  __shared__ float s_depth[kMaxHyp];
  // node cells of the tile, in x order: tile column, ray, 3x3 patch
  __shared__ int s_col[kCostCells];
  __shared__ float s_dir[3][kCostCells];
  __shared__ int s_patch[9][kCostCells];
  __shared__ int s_nodes;
  int lb;
  const JobDesc &J = job_of(B, lb);
  const int D = J.D, F = J.F, W = J.W, H = J.H;
  const int segs = (J.cw + kCostCells - 1) / kCostCells;
  const int cy = lb / segs, cx0 = (lb - cy * segs) * kCostCells;
  const int ncells = min(kCostCells, J.cw - cx0);
  const int tid = threadIdx.x;
  // the job's (deduplicated) slots and the hypothesis depths, once per block
  for (int i = tid; i < F * 12; i += blockDim.x)
    reinterpret_cast<float *>(s_pose)[i] = slot_pose(B, J.slot_base + i / 12)[i % 12];
  for (int i = tid; i < F; i += blockDim.x)
  {
    s_img[i] = slot_image(B, J.slot_base + i);
    s_w[i] = slot_weight(B, J.slot_base + i);
  }
  for (int d = tid; d < D; d += blockDim.x)
    s_depth[d] = A::hyp_depth(J.step, J.min_inv, d);
  const int sd = D + 1;
  for (int i = tid; i < ncells * sd; i += blockDim.x)
    s_out[i] = 0.0f;
  const Cam cam{J.fx, J.fy, J.cx, J.cy};
  if (tid < 32)
  {
    // node test of cell cx0 + tid: quadtree node origin away from the border
    const int x = (cx0 + tid) * 4, y = cy * 4;
    bool node = false;
    if (tid < ncells && x > 0 && y > 0 && x < W - 1 && y < H - 1)
    {
      const int size = 1 << J.levels[(size_t)y * W + x];
      node = x % size == 0 && y % size == 0;
    }
    const unsigned ballot = __ballot_sync(0xffffffffu, node);
    if (node)
    {
      const int k = __popc(ballot & ((1u << tid) - 1u));
      s_col[k] = tid;
      const float3 dir = A::ray((float)x, (float)y, cam);
      s_dir[0][k] = dir.x;
      s_dir[1][k] = dir.y;
      s_dir[2][k] = dir.z;
      const uint8_t *r = J.ref + (size_t)(y - 1) * J.ref_pitch + (x - 1);
#pragma unroll
      for (int jj = 0; jj < 3; ++jj)
#pragma unroll
        for (int ii = 0; ii < 3; ++ii)
          s_patch[3 * jj + ii][k] = __ldg(r + (size_t)jj * J.ref_pitch + ii);
    }
    if (tid == 0)
      s_nodes = __popc(ballot);
  }
  __syncthreads();
  const int n = s_nodes;
  const int pitch = J.slot_pitch;
  // (int)(u + 0.5) in [2, W-2) exactly when u in [1.5, W-2.5) (both bounds
  // are floats, the comparisons exact; NaN fails)
  const float ulo = 1.5f, uhi = (float)W - 2.5f, vhi = (float)H - 2.5f;
  const unsigned bias = 0u - kBias * ((unsigned)pitch + 1u);
  // Thread t evaluates node k = t % n at hypotheses g, g + per, g + 2 per,
  // ... (g = t / n, per = threads per node): consecutive lanes hold
  // neighbouring nodes at one depth, whose projections are neighbours in the
  // slot images.  The node's ray and 3x3 patch stay in registers across the
  // thread's hypotheses and slots.
  const int per = n > 0 ? (int)blockDim.x / n : 0;
  if (n > 0 && tid < per * n)
  {
    const int k = tid % n, g = tid / n;
    const float3 dir = make_float3(s_dir[0][k], s_dir[1][k], s_dir[2][k]);
    unsigned patch[9];
#pragma unroll
    for (int t = 0; t < 9; ++t)
      patch[t] = (unsigned)s_patch[t][k];
    const int col = s_col[k] * sd;
    for (int d = g; d < D; d += per)
    {
      const float3 p = A::scale(dir, s_depth[d]);
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
          // The slot poses are validated as rigid on the host (|r00|+|r01|
          // and |r10|+|r11| <= 1.5), so every patch coordinate + 0.5 lies
          // in [0.5, W-0.5) x [0.5, H-0.5): no clamp needed.
          float px[9], py[9];
          patch_axis(uv.x, T[0], T[1], px);
          patch_axis(uv.y, T[4], T[5], py);
          unsigned s = 0;
#pragma unroll
          for (int t = 0; t < 9; ++t)
          {
            // offset = floor(py+0.5)*pitch + floor(px+0.5), in 32-bit
            // wrap-around arithmetic (the true offset is below 2^31)
            const unsigned hx = round_bits(px[t]);
            const unsigned hy = round_bits(py[t]);
            const unsigned off = hy * (unsigned)pitch + hx + bias;
            s = __usad(patch[t], (unsigned)__ldg(m + off), s);
          }
          const int wgt = s_w[f];
          sad += wgt * (int)s;
          nvalid += wgt;
        }
      }
      const float c = nvalid > 0 ? A::sad_norm((float)sad, (float)nvalid) : 100.0f;
      const int add_num = D; // writer count of the cell (see above)
      s_out[col + d] = A::div(c, (float)add_num);
    }
  }
  __syncthreads();
  // the tile's cells are consecutive in the [cell][D] layout.  Element i is
  // s_out[i + i / D]; i / D = umulhi(i, ceil(2^32 / D)), exact for i < 2^20.
  // D is a multiple of 16, so when the tile starts on a 16-byte boundary
  // (always in the engine's arena; a caller's cost buffer may not) four
  // hypotheses of one cell go out per store.
  float *out = J.lv[0].data + ((size_t)cy * J.cw + cx0) * D;
  const unsigned dinv = 0xffffffffu / (unsigned)D + 1u;
  if ((reinterpret_cast<uintptr_t>(out) & 15u) == 0)
  {
    for (int i4 = tid; i4 < ncells * D / 4; i4 += blockDim.x)
    {
      const int i = 4 * i4;
      const float *src = s_out + i + (int)__umulhi((unsigned)i, dinv);
      reinterpret_cast<float4 *>(out)[i4] = make_float4(src[0], src[1], src[2], src[3]);
    }
  }
  else
  {
    for (int i = tid; i < ncells * D; i += blockDim.x)
      out[i] = s_out[i + (int)__umulhi((unsigned)i, dinv)];
  }
}

} // namespace

int cost_blocks(int cw, int ch) { return ch * ((cw + kCostCells - 1) / kCostCells); }

namespace
{
template <int MINB>
void cost_minb(const Batch &B, int blocks, int arith, size_t sm, cudaStream_t s)
{
  if (arith == QM_ARITH_IEEE)
    k_cost<ArithIeee, MINB><<<blocks, kFlatThreads, sm, s>>>(B);
  else
    k_cost<ArithRef, MINB><<<blocks, kFlatThreads, sm, s>>>(B);
}
} // namespace

void launch_cost(const Batch &B, int blocks, int arith, int max_d, cudaStream_t s,
                 int blocks_per_sm)
{
  const size_t sm = sizeof(float) * kCostCells * (max_d + 1);
  if (blocks_per_sm == 3)
    cost_minb<3>(B, blocks, arith, sm, s);
  else if (blocks_per_sm == 4)
    cost_minb<4>(B, blocks, arith, sm, s);
  else
    cost_minb<5>(B, blocks, arith, sm, s);
}

} // namespace qm
