// Hierarchical min-sum belief propagation and depth extraction
// (bp_extract and its kernels, bpextract.cu:37-395 of the reference).
//
// Layout: per pyramid level, the data cost and the four outgoing-message
// images are [h][w][D] float arrays (hypotheses contiguous, the PIXEL_COST
// layout).  A half-sweep updates the cells of one checkerboard colour in
// place; they only read messages of the other colour, so the update is a
// Jacobi step inside the colour, exactly as the reference's launch.
//
// Lane groups: a cell is handled by a group of LPC lanes (32 for 96 and 128
// hypotheses, 16 for 48 and 64, 8 for 32), so a warp updates 32/LPC cells
// at once; lane g of a group holds hypotheses g, g+LPC, g+2*LPC, ... (3 or
// 4 register slots; every supported count is exactly LPC x slots).  The four
// directions are computed from one load of the data cost and the four
// incoming messages.  The normalising sum uses the reference's stride-halving
// tree (bpextract.cu:293-300) over the next power of two P >= D with zero
// padding: strides >= LPC combine register slots, strides < LPC run as an
// xor butterfly inside the group, so lane 0 of the group ends with the
// bit-identical sum (and, addition being commutative, so does every lane).
// The argmin of the extraction uses the same tree with the reference's tie
// rule (the right element wins only when strictly smaller,
// bpextract.cu:347-355).
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
  static constexpr int P = pow2_ceil(D);              // tree width
  static constexpr int LPC = P / 4 < 32 ? P / 4 : 32; // lanes per cell
  static constexpr int NV = (D + LPC - 1) / LPC;      // register slots per lane
  static constexpr int G = 32 / LPC;                  // cells per warp
  static_assert(NV * LPC == D, "hypothesis count must fill the lane group");
};

// Stride-halving tree sum over the D values of a lane group, held as
// v[k] = value(g + LPC*k).  Strides >= LPC combine register slots (the
// padding beyond D is zero, so those additions are skipped); strides < LPC
// run as an xor butterfly inside the group.  Lane 0 of the group performs
// exactly the reference's additions, and since a + b == b + a bit for bit,
// every lane of the group ends with lane 0's value.
template <int D>
__device__ __forceinline__ float tree_sum(const float (&v)[HypLayout<D>::NV])
{
  constexpr int P = HypLayout<D>::P;
  constexpr int NV = HypLayout<D>::NV;
  constexpr int LPC = HypLayout<D>::LPC;
  float a[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k)
    a[k] = v[k];
#pragma unroll
  for (int s = P / 2; s >= LPC; s /= 2)
  {
    const int t = s / LPC;
#pragma unroll
    for (int k = 0; k < t; ++k)
      if (k + t < NV)
        a[k] += a[k + t];
  }
  float r = a[0];
#pragma unroll
  for (int o = LPC / 2; o > 0; o >>= 1)
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

// minimum over a lane group (exact, order-free)
template <int LPC>
__device__ __forceinline__ float group_min(float v)
{
  if constexpr (LPC == 32)
    return warp_min_redux(v);
  else
  {
#pragma unroll
    for (int o = LPC / 2; o > 0; o >>= 1)
      v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
  }
}

template <int D>
__device__ __forceinline__ void tree_argmin(const float (&v)[HypLayout<D>::NV], int gl,
                                            float &best_v, int &best_i)
{
  constexpr int P = HypLayout<D>::P;
  constexpr int NV = HypLayout<D>::NV;
  constexpr int LPC = HypLayout<D>::LPC;
  float a[NV];
  int ai[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k)
  {
    a[k] = v[k];
    ai[k] = gl + LPC * k;
  }
#pragma unroll
  for (int s = P / 2; s >= LPC; s /= 2)
  {
    const int t = s / LPC;
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
  for (int o = LPC / 2; o > 0; o >>= 1)
  {
    const float ov = __shfl_down_sync(0xffffffffu, r, o, LPC);
    const int oi = __shfl_down_sync(0xffffffffu, ri, o, LPC);
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
// iterations, the cells no sweep reaches.  With two or more iterations the
// batched pipeline does not launch this pass: half-sweeps 0 and 1 copy the
// skipped cells of their own colour (the sweep kernel's `inherit` mode).
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
// bp kernel (bpextract.cu:200-312), one lane group per cell of the active
// colour.  Groups whose cell is skipped or out of range still take part in
// the warp's shuffles (full masks) with zero inputs and store nothing.
//
// msg_load: messages another block of the same launch may have written since
// the launch began are read through L2 (ld.global.cg) by the coarse-level
// kernel below, whose blocks hand messages to each other across cluster
// barriers; the one-launch-per-half-sweep kernel reads them normally.
template <bool L2_ONLY>
__device__ __forceinline__ float msg_load(const float *p)
{
  if constexpr (L2_ONLY)
    return __ldcg(p);
  else
    return *p;
}

// The update of one cell (bp, bpextract.cu:200-312) from its data term and
// its four incoming messages (zeros, and has_* false, where the level ends),
// every lane of the warp taking part (groups without a cell pass zeros):
// for each outgoing direction, emit(dir, m, mean) receives the group's NV
// values m[k] (hypothesis gl + LPC k) and the mean the message subtracts, so
// the message is m[k] - mean.
template <int D, int ARITH, class Emit>
__device__ __forceinline__ void cell_update(const float (&dat)[HypLayout<D>::NV],
                                            const float (&fu)[HypLayout<D>::NV],
                                            const float (&fd)[HypLayout<D>::NV],
                                            const float (&fl)[HypLayout<D>::NV],
                                            const float (&fr)[HypLayout<D>::NV], bool has_u,
                                            bool has_d, bool has_l, bool has_r, const KParams &kp,
                                            int gl, Emit &&emit)
{
  using HL = HypLayout<D>;
  constexpr int NV = HL::NV, LPC = HL::LPC;
  const float P1 = kp.P1, P2 = kp.P2;
  // h of every direction: the data term plus the three other incoming
  // messages, in the reference's order (up, down, left, right skipped as
  // named by the direction); computed up front so the raw inputs die early
  float hall[4][NV];
#pragma unroll
  for (int dir = 0; dir < 4; ++dir)
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
      hall[dir][k] = v;
    }
#pragma unroll
  for (int dir = 0; dir < 4; ++dir)
  {
    const float(&hv)[NV] = hall[dir];
    float lmin = FLT_MAX;
#pragma unroll
    for (int k = 0; k < NV; ++k)
      lmin = fminf(lmin, hv[k]);
    const float hmin = group_min<LPC>(lmin);
    float m[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k)
    {
      const int d = gl + LPC * k;
      // h(d-1): the previous lane's slot k, or for group lane 0 the group's
      // last lane's slot k-1; h(d+1): the next lane's slot k, or for the last
      // lane group lane 0's slot k+1.  One shuffle each, the source lane
      // choosing which register it offers.
      const float up_src = (gl == LPC - 1 && k > 0) ? hv[k > 0 ? k - 1 : 0] : hv[k];
      const float dn_src = (gl == 0 && k + 1 < NV) ? hv[k + 1 < NV ? k + 1 : k] : hv[k];
      const float prev = __shfl_sync(0xffffffffu, up_src, (gl + LPC - 1) & (LPC - 1), LPC);
      const float next = __shfl_sync(0xffffffffu, dn_src, (gl + 1) & (LPC - 1), LPC);
      float mv = hv[k];
      if (d > 0)
        mv = fminf(mv, prev + P1);
      if (d < D - 1)
        mv = fminf(mv, next + P1);
      m[k] = fminf(mv, hmin + P2);
    }
    const float sum = tree_sum<D>(m);
    const float mean = mean_of<D, ARITH>(sum);
    emit(dir, m, mean);
  }
}

// One warp's lane groups of half-sweep `parity` at `level`: items item0 ..
// item0 + G - 1 of the colour's cells (item = y * ceil(w / 2) + x / 2).
template <int D, int ARITH, bool L2_ONLY>
__device__ __forceinline__ void sweep_warp(const JobDesc &J, int level, int parity, int first,
                                           int inherit, const KParams &kp, int item0)
{
  using HL = HypLayout<D>;
  constexpr int NV = HL::NV, LPC = HL::LPC;
  const LevelDesc &L = J.lv[level];
  const int w = L.w, h = L.h, hw = (w + 1) / 2;
  const int lane = threadIdx.x & 31, gl = lane & (LPC - 1);
  const int item = item0 + lane / LPC;
  int x = 0, y = 0;
  bool act = item < hw * h, skipped = false;
  if (act)
  {
    y = item / hw;
    x = 2 * (item - y * hw) + ((y + parity) & 1); // item - y*hw == x / 2
    skipped = x < w && bp_skipped(J, level, x, y, kp.qt_max);
    act = x < w && !skipped;
  }
  if (inherit && skipped)
  {
    // message inheritance of a cell the quadtree test skips at this level:
    // its messages keep the parent's (zeros at the coarsest level), as the
    // reference's copied-down images hold them (bpextract.cu:87-90,374-395);
    // half-sweeps 0 and 1 write them for their colour before any later
    // half-sweep reads them
    const size_t c = (size_t)y * w + x;
    const bool top = level + 1 >= J.nlev;
    const LevelDesc &C = J.lv[top ? level : level + 1];
    const size_t pc = ((size_t)(y >> 1) * C.w + (x >> 1)) * D;
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
      for (int k = 0; k < NV; ++k)
      {
        const int d = gl + LPC * k;
        L.msg[m][c * D + d] = top ? 0.0f : msg_load<L2_ONLY>(C.msg[m] + pc + d);
      }
  }
  if (!__any_sync(0xffffffffu, act))
    return;
  const bool has_u = act && y > 0, has_d = act && y < h - 1;
  const bool has_l = act && x > 0, has_r = act && x < w - 1;
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
    const int d = gl + LPC * k;
    dat[k] = act ? L.data[c * D + d] : 0.0f;
    fu[k] = (ld && has_u) ? msg_load<L2_ONLY>(src_u + d) : 0.0f;
    fd[k] = (ld && has_d) ? msg_load<L2_ONLY>(src_d + d) : 0.0f;
    fl[k] = (ld && has_l) ? msg_load<L2_ONLY>(src_l + d) : 0.0f;
    fr[k] = (ld && has_r) ? msg_load<L2_ONLY>(src_r + d) : 0.0f;
  }
  cell_update<D, ARITH>(dat, fu, fd, fl, fr, has_u, has_d, has_l, has_r, kp, gl,
                        [&](int dir, const float(&m)[NV], float mean) {
                          if (act)
                          {
                            float *out = L.msg[dir] + c * D;
#pragma unroll
                            for (int k = 0; k < NV; ++k)
                              out[gl + LPC * k] = m[k] - mean;
                          }
                        });
}

template <int D, int ARITH>
__global__ void __launch_bounds__(kMaxCellWarps * 32, 4)
    k_bp_sweep(const __grid_constant__ Batch B, int level, int parity, int first, int inherit,
               KParams kp)
{
  constexpr int G = HypLayout<D>::G;
  int lb;
  const JobDesc &J = job_of(B, lb);
  if (J.D != D)
    return;
  const LevelDesc &L = J.lv[level];
  const int hw = (L.w + 1) / 2;
  const int item0 = (lb * (int)(blockDim.x >> 5) + (threadIdx.x >> 5)) * G;
  if (item0 >= hw * L.h)
    return; // the whole warp
  sweep_warp<D, ARITH, false>(J, level, parity, first, inherit, kp, item0);
}

// Every half-sweep of the coarse levels lo..hi (coarse to fine) in one
// launch: a cluster of kCoarseCtas blocks per job walks the levels, each
// half-sweep spread over the cluster's warps, with a cluster barrier (a
// hardware barrier: release / acquire at cluster scope, no spinning) between
// half-sweeps.  A coarse level's costs and messages (about 2.3 MB per
// 752x480 job at levels 2 and 3 together) stay in L2 across its sweeps, and
// its 10 half-sweeps no longer pay a launch and a grid drain each.  The
// arithmetic is the per-half-sweep kernel's (the same device function), so
// the messages are bit-identical; messages are read through L2 because other
// blocks of the cluster wrote them.  Every block of a cluster takes the same
// barriers: the trip counts depend only on the job and the plan.
template <int D, int ARITH>
__global__ void __cluster_dims__(kCoarseCtas, 1, 1) __launch_bounds__(kCoarseThreads, 2)
    k_bp_coarse(const __grid_constant__ Batch B, int j0, CoarsePlan plan, KParams kp)
{
  constexpr int G = HypLayout<D>::G;
  const int job = j0 + (int)blockIdx.x / kCoarseCtas;
  const JobDesc &J = B.jobs ? B.jobs[job] : B.one;
  if (J.D != D)
    return; // the whole cluster
  const int warps = kCoarseThreads / 32;
  const int gw = (int)(blockIdx.x % kCoarseCtas) * warps + (int)(threadIdx.x >> 5);
  const int stride = kCoarseCtas * warps * G;
  for (int level = plan.hi; level >= plan.lo; --level)
  {
    const LevelDesc &L = J.lv[level];
    const int n = (L.w + 1) / 2 * L.h;
    const int iters = plan.iters[level];
    for (int it = 0; it < iters; ++it)
    {
      for (int item0 = gw * G; item0 < n; item0 += stride)
        sweep_warp<D, ARITH, true>(J, level, it & 1, it == 0 ? 1 : 0, it < 2 ? 1 : 0, kp,
                                   item0);
      asm volatile("barrier.cluster.arrive.release.aligned;\n"
                   "barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
    }
  }
}

// ------------------------------------------------------------- extract
// depth_extract (bpextract.cu:314-372), one lane group per level-0 cell.
template <int D, int ARITH>
__global__ void __launch_bounds__(kMaxCellWarps * 32)
    k_extract(const __grid_constant__ Batch B)
{
  using HL = HypLayout<D>;
  constexpr int NV = HL::NV, LPC = HL::LPC, G = HL::G;
  int lb;
  const JobDesc &J = job_of(B, lb);
  if (J.D != D)
    return;
  const LevelDesc &L = J.lv[0];
  const int w = L.w, h = L.h;
  const int lane = threadIdx.x & 31, gl = lane & (LPC - 1);
  const int cell0 = (lb * (int)(blockDim.x >> 5) + (threadIdx.x >> 5)) * G;
  if (cell0 >= w * h)
    return; // the whole warp
  const int cell = cell0 + lane / LPC;
  bool act = cell < w * h;
  int x = 0, y = 0;
  if (act)
  {
    x = cell % w;
    y = cell / w;
    const int lvl = J.levels[(size_t)min(y * 4, J.H - 1) * J.W + min(x * 4, J.W - 1)];
    const int size = 1 << lvl;
    if ((x * 4) % size != 0 || (y * 4) % size != 0)
    {
      if (gl == 0 && J.labels)
        J.labels[cell] = -1;
      act = false;
    }
  }
  if (!__any_sync(0xffffffffu, act))
    return;
  const size_t c = (size_t)cell;
  float b[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k)
  {
    const int d = gl + LPC * k;
    float v = 0.0f;
    if (act)
    {
      v = L.data[c * D + d];
      if (x != 0)
        v += L.msg[kRight][(c - 1) * D + d];
      if (x != w - 1)
        v += L.msg[kLeft][(c + 1) * D + d];
      if (y != 0)
        v += L.msg[kDown][(c - w) * D + d];
      if (y != h - 1)
        v += L.msg[kUp][(c + w) * D + d];
    }
    b[k] = v;
  }
  float bmin;
  int best;
  tree_argmin<D>(b, gl, bmin, best);
  best = __shfl_sync(0xffffffffu, best, 0, LPC);
  bmin = __shfl_sync(0xffffffffu, bmin, 0, LPC);
  // neighbours of the winner for the parabola
  const int ip = best > 0 ? best - 1 : 0, in_ = best < D - 1 ? best + 1 : D - 1;
  float pre = 0.0f, post = 0.0f;
#pragma unroll
  for (int k = 0; k < NV; ++k)
  {
    const float vp = __shfl_sync(0xffffffffu, b[k], ip % LPC, LPC);
    const float vn = __shfl_sync(0xffffffffu, b[k], in_ % LPC, LPC);
    if (ip / LPC == k)
      pre = vp;
    if (in_ / LPC == k)
      post = vn;
  }
  if (gl != 0 || !act)
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
void sweep_d(const Batch &B, int blocks, int level, int parity, int first, int inherit,
             KParams kp, int arith, int warps, cudaStream_t s)
{
  if (arith == QM_ARITH_IEEE)
    k_bp_sweep<D, QM_ARITH_IEEE>
        <<<blocks, warps * 32, 0, s>>>(B, level, parity, first, inherit, kp);
  else
    k_bp_sweep<D, QM_ARITH_REFERENCE>
        <<<blocks, warps * 32, 0, s>>>(B, level, parity, first, inherit, kp);
}

template <int D>
void coarse_d(const Batch &B, int j0, int jobs, const CoarsePlan &plan, KParams kp, int arith,
              cudaStream_t s)
{
  if (arith == QM_ARITH_IEEE)
    k_bp_coarse<D, QM_ARITH_IEEE><<<jobs * kCoarseCtas, kCoarseThreads, 0, s>>>(B, j0, plan, kp);
  else
    k_bp_coarse<D, QM_ARITH_REFERENCE>
        <<<jobs * kCoarseCtas, kCoarseThreads, 0, s>>>(B, j0, plan, kp);
}

template <int D>
void extract_d(const Batch &B, int blocks, int arith, int warps, cudaStream_t s)
{
  if (arith == QM_ARITH_IEEE)
    k_extract<D, QM_ARITH_IEEE><<<blocks, warps * 32, 0, s>>>(B);
  else
    k_extract<D, QM_ARITH_REFERENCE><<<blocks, warps * 32, 0, s>>>(B);
}

} // namespace

bool bp_supported_d(int d) { return d == 32 || d == 48 || d == 64 || d == 96 || d == 128; }

int bp_cells_per_warp(int d)
{
  switch (d)
  {
  case 32: return HypLayout<32>::G;
  case 48: return HypLayout<48>::G;
  case 64: return HypLayout<64>::G;
  case 96: return HypLayout<96>::G;
  case 128: return HypLayout<128>::G;
  default: return 1;
  }
}

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
namespace
{
void sweep_any(const Batch &B, int blocks, int d, int level, int parity, int first, int inherit,
               KParams kp, int arith, int warps, cudaStream_t s)
{
  switch (d)
  {
  case 32: sweep_d<32>(B, blocks, level, parity, first, inherit, kp, arith, warps, s); break;
  case 48: sweep_d<48>(B, blocks, level, parity, first, inherit, kp, arith, warps, s); break;
  case 64: sweep_d<64>(B, blocks, level, parity, first, inherit, kp, arith, warps, s); break;
  case 96: sweep_d<96>(B, blocks, level, parity, first, inherit, kp, arith, warps, s); break;
  case 128: sweep_d<128>(B, blocks, level, parity, first, inherit, kp, arith, warps, s); break;
  default: break;
  }
}
} // namespace

void launch_bp_sweep(const Batch &B, int blocks, int d, int level, int it, KParams kp, int arith,
                     cudaStream_t s, int warps, int inherit)
{
  sweep_any(B, blocks, d, level, it & 1, it == 0 ? 1 : 0, inherit && it < 2 ? 1 : 0, kp, arith,
            warps, s);
}

void launch_bp_sweep_own(const Batch &B, int blocks, int d, int level, int parity, KParams kp,
                         int arith, cudaStream_t s, int warps)
{
  sweep_any(B, blocks, d, level, parity, 0, 0, kp, arith, warps, s);
}

void launch_bp_coarse(const Batch &B, int j0, int jobs, int d, const CoarsePlan &plan,
                      KParams kp, int arith, cudaStream_t s)
{
  switch (d)
  {
  case 32: coarse_d<32>(B, j0, jobs, plan, kp, arith, s); break;
  case 48: coarse_d<48>(B, j0, jobs, plan, kp, arith, s); break;
  case 64: coarse_d<64>(B, j0, jobs, plan, kp, arith, s); break;
  case 96: coarse_d<96>(B, j0, jobs, plan, kp, arith, s); break;
  case 128: coarse_d<128>(B, j0, jobs, plan, kp, arith, s); break;
  default: break;
  }
}

void launch_extract(const Batch &B, int blocks, int d, int arith, cudaStream_t s, int warps)
{
  switch (d)
  {
  case 32: extract_d<32>(B, blocks, arith, warps, s); break;
  case 48: extract_d<48>(B, blocks, arith, warps, s); break;
  case 64: extract_d<64>(B, blocks, arith, warps, s); break;
  case 96: extract_d<96>(B, blocks, arith, warps, s); break;
  case 128: extract_d<128>(B, blocks, arith, warps, s); break;
  default: break;
  }
}

} // namespace qm
