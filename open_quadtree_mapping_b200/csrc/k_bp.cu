// Hierarchical min-sum belief propagation and depth extraction
// (bp_extract and its kernels, bpextract.cu:37-395 of the reference).
//
// Layout: per pyramid level, the data cost and the four outgoing-message
// images are [h][w][D] float arrays (hypotheses contiguous, the PIXEL_COST
// layout).  A half-sweep updates the cells of one checkerboard colour in
// place; they only read messages of the other colour, so the update is a
// Jacobi step inside the colour, exactly as the reference's launch.
//
// Warp-per-cell: lane l holds hypotheses l, l+32, l+64, ... of the cell.  The
// four directions are computed from one load of the data cost and the four
// incoming messages.  The normalising sum uses the reference's stride-halving
// tree (bpextract.cu:293-300): strides >= 32 combine register slots, strides
// 16..1 use __shfl_down, so lane 0 ends with the bit-identical sum.  The
// argmin of the extraction uses the same tree with the reference's tie rule
// (the right element wins only when strictly smaller, bpextract.cu:347-355).
// Hypothesis counts that are not a power of two run the tree over the next
// power of two with neutral padding (0 for sums, +inf for minima).
//
// Bytes per updated cell and half-sweep: 9*D*4 (data + 4 messages read, 4
// messages written).
#include <cfloat>

#include "launch.h"

namespace qm
{

namespace
{

constexpr __host__ __device__ int pow2_ceil(int n)
{
  int p = 1;
  while (p < n)
    p <<= 1;
  return p;
}

template <int D>
struct HypLayout
{
  static constexpr int NV = (D + 31) / 32; // register slots per lane
  static constexpr int P = pow2_ceil(D);   // tree width
};

// Stride-halving tree sum over D values held as v[k] = value(lane + 32k).
// Strides >= 32 combine register slots; strides 16..1 run as an xor
// butterfly.  Lane 0 performs exactly the reference's additions, and since
// a + b == b + a bit for bit, every lane ends with lane 0's value, so no
// broadcast is needed.
template <int D>
__device__ __forceinline__ float tree_sum(float (&v)[HypLayout<D>::NV])
{
  constexpr int P = HypLayout<D>::P;
  constexpr int NV = HypLayout<D>::NV;
  float a[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k)
    a[k] = v[k];
#pragma unroll
  for (int s = P / 2; s >= 32; s /= 2)
  {
    const int t = s / 32;
#pragma unroll
    for (int k = 0; k < t; ++k)
      if (k + t < NV)
        a[k] += a[k + t];
  }
  float r = a[0];
#pragma unroll
  for (int o = (P / 2 < 16 ? P / 2 : 16); o > 0; o >>= 1)
    r += __shfl_xor_sync(0xffffffffu, r, o);
  return r;
}

// Order-preserving map between floats and signed ints (an involution), so a
// float minimum can use the integer warp reduction.
__device__ __forceinline__ int order_key(float f)
{
  const int b = __float_as_int(f);
  return b ^ ((b >> 31) & 0x7fffffff);
}

__device__ __forceinline__ float warp_min_redux(float v)
{
  const int k = __reduce_min_sync(0xffffffffu, order_key(v));
  return __int_as_float(k ^ ((k >> 31) & 0x7fffffff));
}

template <int D>
__device__ __forceinline__ void tree_argmin(const float (&v)[HypLayout<D>::NV], int lane,
                                            float &best_v, int &best_i)
{
  constexpr int P = HypLayout<D>::P;
  constexpr int NV = HypLayout<D>::NV;
  float a[NV];
  int ai[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k)
  {
    a[k] = v[k];
    ai[k] = lane + 32 * k;
  }
#pragma unroll
  for (int s = P / 2; s >= 32; s /= 2)
  {
    const int t = s / 32;
#pragma unroll
    for (int k = 0; k < t; ++k)
      if (k + t < NV && a[k + t] < a[k])
      {
        a[k] = a[k + t];
        ai[k] = ai[k + t];
      }
  }
  float r = a[0];
  int ri = ai[0];
#pragma unroll
  for (int o = (P / 2 < 16 ? P / 2 : 16); o > 0; o >>= 1)
  {
    const float ov = __shfl_down_sync(0xffffffffu, r, o);
    const int oi = __shfl_down_sync(0xffffffffu, ri, o);
    if (ov < r)
    {
      r = ov;
      ri = oi;
    }
  }
  best_v = r;
  best_i = ri;
}

// sum / (float)DEPTH_NUM (bpextract.cu:302); D is a compile-time constant
// here as DEPTH_NUM is in the reference.
template <int D, int ARITH>
__device__ __forceinline__ float mean_of(float sum)
{
  if (ARITH == QM_ARITH_IEEE)
    return __fdiv_rn(sum, (float)D);
  return sum / (float)D;
}

// The three kernels below move whole float4 groups of hypotheses (D is a
// multiple of 16 for every supported count, and every cell row starts on a
// 16-byte boundary); each component keeps its own arithmetic.

// ------------------------------------------------------------- pyramid
// cost_distribute (bpextract.cu:169-198): L_l(x,y) = sum of the existing 2x2
// children, x offset outer, y offset inner, starting from 0.
__global__ void __launch_bounds__(kFlatThreads)
    k_pyramid(const __grid_constant__ Batch B, int level)
{
  int lb;
  const JobDesc &J = job_of(B, lb);
  const LevelDesc &Lf = J.lv[level - 1];
  const LevelDesc &Lc = J.lv[level];
  const int D4 = J.D / 4;
  const long t = (long)lb * blockDim.x + threadIdx.x;
  if (t >= (long)Lc.w * Lc.h * D4)
    return;
  const int cell = (int)(t / D4);
  const int q = (int)(t - (long)cell * D4);
  const int x = cell % Lc.w, y = cell / Lc.w;
  const float4 *src = reinterpret_cast<const float4 *>(Lf.data);
  float4 s = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int jj = 0; jj < 2; ++jj)
      if (2 * x + i < Lf.w && 2 * y + jj < Lf.h)
      {
        const float4 v = src[((size_t)(2 * y + jj) * Lf.w + (2 * x + i)) * D4 + q];
        s.x += v.x;
        s.y += v.y;
        s.z += v.z;
        s.w += v.w;
      }
  reinterpret_cast<float4 *>(Lc.data)[(size_t)cell * D4 + q] = s;
}

// The reference's quadtree test of the bp kernel (bpextract.cu:214-220): a
// cell of level l is left alone by every sweep of that level when the
// quadtree level at the sample pixel of its pre-checkerboard column (x / 2)
// exceeds l + 2.
__device__ __forceinline__ bool bp_skipped(const JobDesc &J, int level, int x, int y, int qt_max)
{
  const int ilev = level + 2;
  if (ilev > qt_max)
    return false;
  const int size = 1 << ilev;
  const int sx = min((x >> 1) * size, J.W - 1), sy = min(y * size, J.H - 1);
  return (int)J.levels[(size_t)sy * J.W + sx] > ilev;
}

// Message inheritance.  The reference starts every level from a copy of the
// parent messages (upsample, bpextract.cu:374-395), or from zeros at the
// coarsest level (bpextract.cu:87-90), and then sweeps.  Most of those copies
// are never read: the first half-sweep reads the parents directly (the sweep
// kernel's `first` mode), and every cell the sweeps update overwrites its
// copy before anyone reads it.  The copies that ARE read later are written
// here: cells the quadtree test skips at this level, and, with fewer than two
// iterations, the cells no sweep reaches.
__global__ void __launch_bounds__(kFlatThreads)
    k_msg_inherit(const __grid_constant__ Batch B, int level, int iters, int qt_max)
{
  int lb;
  const JobDesc &J = job_of(B, lb);
  const LevelDesc &F = J.lv[level];
  const int D4 = J.D / 4;
  const long t = (long)lb * blockDim.x + threadIdx.x;
  if (t >= (long)F.w * F.h * D4)
    return;
  const int cell = (int)(t / D4);
  const int q = (int)(t - (long)cell * D4);
  const int x = cell % F.w, y = cell / F.w;
  // iteration i updates the cells with x + y + i even
  const bool needed = iters <= 0 || (iters == 1 && ((x + y) & 1)) ||
                      bp_skipped(J, level, x, y, qt_max);
  if (!needed)
    return;
  if (level + 1 < J.nlev)
  {
    const LevelDesc &C = J.lv[level + 1];
    const size_t src = ((size_t)(y >> 1) * C.w + (x >> 1)) * D4 + q;
#pragma unroll
    for (int m = 0; m < 4; ++m)
      reinterpret_cast<float4 *>(F.msg[m])[t] = reinterpret_cast<const float4 *>(C.msg[m])[src];
  }
  else
  {
#pragma unroll
    for (int m = 0; m < 4; ++m)
      reinterpret_cast<float4 *>(F.msg[m])[t] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  }
}

// ------------------------------------------------------------- sweep
// bp kernel (bpextract.cu:200-312), one warp per cell of the active colour.
template <int D, int ARITH>
__global__ void __launch_bounds__(kCellWarps * 32)
    k_bp_sweep(const __grid_constant__ Batch B, int level, int parity, int first, KParams kp)
{
  constexpr int NV = HypLayout<D>::NV;
  int lb;
  const JobDesc &J = job_of(B, lb);
  if (J.D != D)
    return;
  const LevelDesc &L = J.lv[level];
  const int w = L.w, h = L.h, hw = (w + 1) / 2;
  const int warp = lb * kCellWarps + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (warp >= hw * h)
    return;
  const int y = warp / hw, bx = warp - y * hw;
  const int x = 2 * bx + ((y + parity) & 1); // bx == x / 2
  if (x >= w || bp_skipped(J, level, x, y, kp.qt_max))
    return;
  const bool has_u = y > 0, has_d = y < h - 1, has_l = x > 0, has_r = x < w - 1;
  const size_t c = (size_t)y * w + x;

  // Incoming messages: the neighbours' own ones, or in the first half-sweep
  // of a level the ones their parents ended with (0 at the coarsest level),
  // which is what the reference's copied-down messages hold at that point.
  const float *src_u = nullptr, *src_d = nullptr, *src_l = nullptr, *src_r = nullptr;
  if (!first)
  {
    src_u = L.msg[kDown] + (c - w) * D;
    src_d = L.msg[kUp] + (c + w) * D;
    src_l = L.msg[kRight] + (c - 1) * D;
    src_r = L.msg[kLeft] + (c + 1) * D;
  }
  else if (level + 1 < J.nlev)
  {
    const LevelDesc &C = J.lv[level + 1];
    auto parent = [&](int xn, int yn) { return ((size_t)(yn >> 1) * C.w + (xn >> 1)) * D; };
    src_u = C.msg[kDown] + parent(x, y - 1);
    src_d = C.msg[kUp] + parent(x, y + 1);
    src_l = C.msg[kRight] + parent(x - 1, y);
    src_r = C.msg[kLeft] + parent(x + 1, y);
  }
  const bool ld = src_u != nullptr;

  float dat[NV], fu[NV], fd[NV], fl[NV], fr[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k)
  {
    const int d = lane + 32 * k;
    const bool in = d < D;
    dat[k] = in ? L.data[c * D + d] : 0.0f;
    fu[k] = (in && ld && has_u) ? src_u[d] : 0.0f;
    fd[k] = (in && ld && has_d) ? src_d[d] : 0.0f;
    fl[k] = (in && ld && has_l) ? src_l[d] : 0.0f;
    fr[k] = (in && ld && has_r) ? src_r[d] : 0.0f;
  }
  const float P1 = kp.P1, P2 = kp.P2;
#pragma unroll
  for (int dir = 0; dir < 4; ++dir)
  {
    float hv[NV];
    float lmin = FLT_MAX;
#pragma unroll
    for (int k = 0; k < NV; ++k)
    {
      float v = dat[k];
      if (dir != kUp && has_u)
        v += fu[k];
      if (dir != kDown && has_d)
        v += fd[k];
      if (dir != kLeft && has_l)
        v += fl[k];
      if (dir != kRight && has_r)
        v += fr[k];
      const bool in = lane + 32 * k < D;
      hv[k] = in ? v : FLT_MAX;
      lmin = fminf(lmin, hv[k]);
    }
    const float hmin = warp_min_redux(lmin);
    float m[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k)
    {
      const int d = lane + 32 * k;
      // h(d-1): lane-1's slot k, or for lane 0 lane 31's slot k-1; h(d+1):
      // lane+1's slot k, or for lane 31 lane 0's slot k+1.  One shuffle each,
      // the source lane choosing which register it offers.
      const float up_src = (lane == 31 && k > 0) ? hv[k > 0 ? k - 1 : 0] : hv[k];
      const float dn_src = (lane == 0 && k + 1 < NV) ? hv[k + 1 < NV ? k + 1 : k] : hv[k];
      const float prev = __shfl_sync(0xffffffffu, up_src, (lane + 31) & 31);
      const float next = __shfl_sync(0xffffffffu, dn_src, (lane + 1) & 31);
      float mv = hv[k];
      if (d > 0)
        mv = fminf(mv, prev + P1);
      if (d < D - 1)
        mv = fminf(mv, next + P1);
      mv = fminf(mv, hmin + P2);
      m[k] = d < D ? mv : 0.0f;
    }
    const float sum = tree_sum<D>(m);
    const float mean = mean_of<D, ARITH>(sum);
    float *out = L.msg[dir] + c * D;
#pragma unroll
    for (int k = 0; k < NV; ++k)
    {
      const int d = lane + 32 * k;
      if (d < D)
        out[d] = m[k] - mean;
    }
  }
}

// ------------------------------------------------------------- extract
// depth_extract (bpextract.cu:314-372), one warp per level-0 cell.
template <int D, int ARITH>
__global__ void __launch_bounds__(kCellWarps * 32)
    k_extract(const __grid_constant__ Batch B)
{
  constexpr int NV = HypLayout<D>::NV;
  int lb;
  const JobDesc &J = job_of(B, lb);
  if (J.D != D)
    return;
  const LevelDesc &L = J.lv[0];
  const int w = L.w, h = L.h;
  const int cell = lb * kCellWarps + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (cell >= w * h)
    return;
  const int x = cell % w, y = cell / w;
  const int lvl = J.levels[(size_t)min(y * 4, J.H - 1) * J.W + min(x * 4, J.W - 1)];
  const int size = 1 << lvl;
  if ((x * 4) % size != 0 || (y * 4) % size != 0)
  {
    if (lane == 0 && J.labels)
      J.labels[cell] = -1;
    return;
  }
  const size_t c = (size_t)cell;
  float b[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k)
  {
    const int d = lane + 32 * k;
    if (d < D)
    {
      float v = L.data[c * D + d];
      if (x != 0)
        v += L.msg[kRight][(c - 1) * D + d];
      if (x != w - 1)
        v += L.msg[kLeft][(c + 1) * D + d];
      if (y != 0)
        v += L.msg[kDown][(c - w) * D + d];
      if (y != h - 1)
        v += L.msg[kUp][(c + w) * D + d];
      b[k] = v;
    }
    else
    {
      b[k] = __int_as_float(0x7f800000); // +inf padding
    }
  }
  float bmin;
  int best;
  tree_argmin<D>(b, lane, bmin, best);
  best = __shfl_sync(0xffffffffu, best, 0);
  bmin = __shfl_sync(0xffffffffu, bmin, 0);
  // neighbours of the winner for the parabola
  const int ip = best > 0 ? best - 1 : 0, in_ = best < D - 1 ? best + 1 : D - 1;
  float pre = 0.0f, post = 0.0f;
#pragma unroll
  for (int k = 0; k < NV; ++k)
  {
    const float vp = __shfl_sync(0xffffffffu, b[k], ip & 31);
    const float vn = __shfl_sync(0xffffffffu, b[k], in_ & 31);
    if ((ip >> 5) == k)
      pre = vp;
    if ((in_ >> 5) == k)
      post = vn;
  }
  if (lane != 0)
    return;
  float disparity = (float)best;
  if (best > 0 && best < D - 1)
  {
    if (ARITH == QM_ARITH_IEEE)
    {
      const float a = __fadd_rn(__fsub_rn(pre, __fmul_rn(2.0f, bmin)), post);
      const float bb = __fadd_rn(-pre, post);
      const float b_a = __fdiv_rn(bb, a);
      if (isfinite(b_a))
        disparity = __fsub_rn((float)best, __fdiv_rn(b_a, 2.0f));
    }
    else
    {
      const float a = pre - 2.0f * bmin + post;
      const float bb = -pre + post;
      const float b_a = bb / a;
      if (isfinite(b_a))
        disparity = (float)best - b_a / 2.0f;
    }
  }
  float depth;
  if (ARITH == QM_ARITH_IEEE)
    depth = (float)__ddiv_rn(1.0, __dadd_rn(__dmul_rn(J.step, (double)disparity), J.min_inv));
  else
    depth = 1.0 / (J.step * disparity + J.min_inv);
  J.sparse[(size_t)(y * 4) * J.W + x * 4] = depth;
  if (J.labels)
    J.labels[cell] = best;
}

template <int D>
void sweep_d(const Batch &B, int blocks, int level, int it, KParams kp, int arith,
             cudaStream_t s)
{
  const int parity = it & 1, first = it == 0 ? 1 : 0;
  if (arith == QM_ARITH_IEEE)
    k_bp_sweep<D, QM_ARITH_IEEE><<<blocks, kCellWarps * 32, 0, s>>>(B, level, parity, first, kp);
  else
    k_bp_sweep<D, QM_ARITH_REFERENCE><<<blocks, kCellWarps * 32, 0, s>>>(B, level, parity, first,
                                                                         kp);
}

template <int D>
void extract_d(const Batch &B, int blocks, int arith,
               cudaStream_t s)
{
  if (arith == QM_ARITH_IEEE)
    k_extract<D, QM_ARITH_IEEE><<<blocks, kCellWarps * 32, 0, s>>>(B);
  else
    k_extract<D, QM_ARITH_REFERENCE><<<blocks, kCellWarps * 32, 0, s>>>(B);
}

} // namespace

bool bp_supported_d(int d) { return d == 32 || d == 48 || d == 64 || d == 96 || d == 128; }

void launch_pyramid(const Batch &B, int blocks, int level,
                    cudaStream_t s)
{
  k_pyramid<<<blocks, kFlatThreads, 0, s>>>(B, level);
}

void launch_msg_inherit(const Batch &B, int blocks, int level, int iters, int qt_max,
                        cudaStream_t s)
{
  k_msg_inherit<<<blocks, kFlatThreads, 0, s>>>(B, level, iters, qt_max);
}

// A batch with mixed hypothesis counts launches one sweep per count present;
// each launch skips the jobs of other counts.
void launch_bp_sweep(const Batch &B, int blocks, int d, int level, int it, KParams kp, int arith,
                     cudaStream_t s)
{
  switch (d)
  {
  case 32: sweep_d<32>(B, blocks, level, it, kp, arith, s); break;
  case 48: sweep_d<48>(B, blocks, level, it, kp, arith, s); break;
  case 64: sweep_d<64>(B, blocks, level, it, kp, arith, s); break;
  case 96: sweep_d<96>(B, blocks, level, it, kp, arith, s); break;
  case 128: sweep_d<128>(B, blocks, level, it, kp, arith, s); break;
  default: break;
  }
}

void launch_extract(const Batch &B, int blocks, int d,
                    int arith, cudaStream_t s)
{
  switch (d)
  {
  case 32: extract_d<32>(B, blocks, arith, s); break;
  case 48: extract_d<48>(B, blocks, arith, s); break;
  case 64: extract_d<64>(B, blocks, arith, s); break;
  case 96: extract_d<96>(B, blocks, arith, s); break;
  case 128: extract_d<128>(B, blocks, arith, s); break;
  default: break;
  }
}

} // namespace qm
