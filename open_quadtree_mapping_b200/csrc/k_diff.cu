// Differentiable path (the training-side pattern of the pipeline): a
// temperature-softened BP belief readout and the adjoints of the BP
// half-sweeps, of an edge-aware upsampling with per-pixel weight factors, and
// of the fusion update.  The product path keeps the hard argmin; these
// kernels serve parameter fitting (BP penalties P1, P2 and the upsampling
// weight factors) against ground-truth depth.
//
// Soft readout, per node cell (the node test of depth_extract,
// bpextract.cu:314-372): beliefs b(d) = data + the four incoming messages in
// the extraction's order, p(d) = softmax(-b(d)/tau), disparity = sum p(d) d,
// depth = 1 / (step * disparity + min) (FP64).
//
// BP adjoint.  A half-sweep writes, for every updated cell c and direction,
// m(d) = min(h(d), h(d-1)+P1, h(d+1)+P1, min_k h(k)+P2) - mean_d(...), where h
// is the data term plus three incoming messages.  Reverse mode follows the
// selected term of each minimum (ties go to the earliest candidate, the
// forward's order) and subtracts the mean of the adjoint.  The adjoint state
// A holds dL/d(message) for every cell and direction; the backward of a
// half-sweep consumes A at the cells it updated (their earlier values were
// overwritten, so A restarts at 0 there) and adds to A at the neighbours'
// messages those cells read, each written by exactly one cell (no atomics).
// dL/dP1 and dL/dP2 are accumulated in FP64.  Messages are recomputed per
// level from the level's starting state (the parents' final messages) instead
// of being stored for the whole pyramid.
//
// Weighted upsampling: the row and column systems of global_upsample
// (depth_upsample.cu:20-302) with every inner edge weight multiplied by a
// per-pixel factor omega (the edge between a pixel and its left / upper
// neighbour takes that pixel's factor), solved per line in FP64 by the Thomas
// algorithm.  The systems are symmetric, so the adjoint solve is the same
// solve; dL/dw for the edge (k-1, k) is -lambda (g(k) - g(k-1)) (s(k) -
// s(k-1)) summed over the two right-hand sides.
//
// Fusion adjoint: the update of fuse_currentmap evaluated on dual numbers
// (value, derivative with respect to the upsampled depth).
#include <cfloat>
#include <type_traits>

#include "launch.h"

namespace qm
{

namespace
{

constexpr int kDiffWarps = 8;

// Arithmetic of a real type: float for the product path, double for the
// gradient-check mode.
template <class R>
struct Real;
template <>
struct Real<float>
{
  static __device__ __forceinline__ float big() { return FLT_MAX; }
  static __device__ __forceinline__ float min(float a, float b) { return fminf(a, b); }
  static __device__ __forceinline__ float exp(float a) { return expf(a); }
};
template <>
struct Real<double>
{
  static __device__ __forceinline__ double big() { return DBL_MAX; }
  static __device__ __forceinline__ double min(double a, double b) { return fmin(a, b); }
  static __device__ __forceinline__ double exp(double a) { return ::exp(a); }
};

template <class R>
__device__ __forceinline__ R warp_sum(R v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <class R>
__device__ __forceinline__ R warp_min(R v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v = Real<R>::min(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// value at hypothesis d-1 / d+1 of a per-lane register array (lane l holds
// d = l + 32k), one shuffle per register; lanes at the ends of the range get
// their own value back (callers mask them)
template <int NV, class R>
__device__ __forceinline__ void neighbours(const R (&v)[NV], int lane, int k, R &prev, R &next)
{
  const R up_src = (lane == 31 && k > 0) ? v[k > 0 ? k - 1 : 0] : v[k];
  const R dn_src = (lane == 0 && k + 1 < NV) ? v[k + 1 < NV ? k + 1 : k] : v[k];
  prev = __shfl_sync(0xffffffffu, up_src, (lane + 31) & 31);
  next = __shfl_sync(0xffffffffu, dn_src, (lane + 1) & 31);
}

template <class R>
__device__ __forceinline__ bool skipped(const DiffBpR<R> &a, int x, int y)
{
  const int ilev = a.level + 2;
  if (ilev > a.qt_max)
    return false;
  const int size = 1 << ilev;
  const int sx = min((x >> 1) * size, a.W - 1), sy = min(y * size, a.H - 1);
  return (int)a.levels[(size_t)sy * a.W + sx] > ilev;
}

template <class R>
__device__ __forceinline__ bool is_node(const DiffBpR<R> &a, int x, int y)
{
  const int lvl = a.levels[(size_t)min(y * 4, a.H - 1) * a.W + min(x * 4, a.W - 1)];
  const int size = 1 << lvl;
  return (x * 4) % size == 0 && (y * 4) % size == 0;
}

// ------------------------------------------------------------ soft readout
template <int D, class R>
__global__ void __launch_bounds__(kDiffWarps * 32)
    k_soft_readout(const DiffBpR<R> a, int backward)
{
  using M = Real<R>;
  constexpr int NV = (D + 31) / 32;
  const int cell = blockIdx.x * kDiffWarps + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const int w = a.w, h = a.h;
  if (cell >= w * h)
    return;
  const int x = cell % w, y = cell / w;
  if (!is_node(a, x, y))
    return;
  const size_t c = (size_t)cell;
  R b[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k)
  {
    const int d = lane + 32 * k;
    R v = M::big();
    if (d < D)
    {
      v = a.data[c * D + d];
      if (x != 0)
        v += a.S[kRight][(c - 1) * D + d];
      if (x != w - 1)
        v += a.S[kLeft][(c + 1) * D + d];
      if (y != 0)
        v += a.S[kDown][(c - w) * D + d];
      if (y != h - 1)
        v += a.S[kUp][(c + w) * D + d];
    }
    b[k] = v;
  }
  R lmin = M::big();
#pragma unroll
  for (int k = 0; k < NV; ++k)
    lmin = M::min(lmin, b[k]);
  const R bmin = warp_min<R>(lmin);
  const R tau = (R)a.tau;
  R e[NV], z = 0, s = 0;
#pragma unroll
  for (int k = 0; k < NV; ++k)
  {
    const int d = lane + 32 * k;
    e[k] = d < D ? M::exp(-(b[k] - bmin) / tau) : (R)0;
    z += e[k];
    s += e[k] * (R)d;
  }
  z = warp_sum<R>(z);
  s = warp_sum<R>(s);
  const R disp = s / z;
  const double depth = 1.0 / (a.step * (double)disp + a.min_inv);
  const size_t px = (size_t)(y * 4) * a.W + x * 4;
  if (!backward)
  {
    if (lane == 0)
      a.sparse[px] = (float)depth;
    return;
  }
  const float g = a.g_sparse[px];
  if (g == 0.0f)
    return;
  // d depth / d disparity = -step * depth^2; d disparity / d b(d) =
  // -(1/tau) p(d) (d - disparity)
  const R g_disp = (R)(-a.step * depth * depth * (double)g);
#pragma unroll
  for (int k = 0; k < NV; ++k)
  {
    const int d = lane + 32 * k;
    if (d >= D)
      continue;
    const R gb = g_disp * (-(e[k] / z) * ((R)d - disp) / tau);
    if (x != 0)
      a.A[kRight][(c - 1) * D + d] += gb;
    if (x != w - 1)
      a.A[kLeft][(c + 1) * D + d] += gb;
    if (y != 0)
      a.A[kDown][(c - w) * D + d] += gb;
    if (y != h - 1)
      a.A[kUp][(c + w) * D + d] += gb;
  }
}

// ------------------------------------------------------------ BP adjoint
template <int D, class R>
__global__ void __launch_bounds__(kDiffWarps * 32) k_bp_sweep_bwd(const DiffBpR<R> a)
{
  using M = Real<R>;
  constexpr int NV = (D + 31) / 32;
  const int lane = threadIdx.x & 31;
  const int w = a.w, h = a.h, hw = (w + 1) / 2;
  const int item = blockIdx.x * kDiffWarps + (threadIdx.x >> 5);
  if (item >= hw * h)
    return;
  const int y = item / hw;
  const int x = 2 * (item - y * hw) + ((y + a.parity) & 1);
  if (x >= w || skipped(a, x, y))
    return;
  const bool has_u = y > 0, has_d = y < h - 1, has_l = x > 0, has_r = x < w - 1;
  const size_t c = (size_t)y * w + x;
  R dat[NV], fu[NV], fd[NV], fl[NV], fr[NV];
  R gu[NV], gd[NV], gl[NV], gr[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k)
  {
    const int d = lane + 32 * k;
    const bool in = d < D;
    dat[k] = in ? a.data[c * D + d] : (R)0;
    fu[k] = (in && has_u) ? a.S[kDown][(c - w) * D + d] : (R)0;
    fd[k] = (in && has_d) ? a.S[kUp][(c + w) * D + d] : (R)0;
    fl[k] = (in && has_l) ? a.S[kRight][(c - 1) * D + d] : (R)0;
    fr[k] = (in && has_r) ? a.S[kLeft][(c + 1) * D + d] : (R)0;
    gu[k] = gd[k] = gl[k] = gr[k] = (R)0;
  }
  const R P1 = (R)a.P1, P2 = (R)a.P2;
  R gp1 = 0, gp2 = 0;
#pragma unroll
  for (int dir = 0; dir < 4; ++dir)
  {
    R hv[NV];
    R lmin = M::big();
#pragma unroll
    for (int k = 0; k < NV; ++k)
    {
      R v = dat[k];
      if (dir != kUp && has_u)
        v += fu[k];
      if (dir != kDown && has_d)
        v += fd[k];
      if (dir != kLeft && has_l)
        v += fl[k];
      if (dir != kRight && has_r)
        v += fr[k];
      hv[k] = (lane + 32 * k < D) ? v : M::big();
      lmin = M::min(lmin, hv[k]);
    }
    const R hmin = warp_min<R>(lmin);
    // the first hypothesis attaining the minimum
    int amin = D;
#pragma unroll
    for (int k = NV - 1; k >= 0; --k)
    {
      const unsigned bal = __ballot_sync(0xffffffffu, hv[k] == hmin);
      if (bal)
        amin = 32 * k + __ffs(bal) - 1;
    }
    // adjoint of the outgoing message, minus its mean
    R gm[NV], gsum = 0;
#pragma unroll
    for (int k = 0; k < NV; ++k)
    {
      const int d = lane + 32 * k;
      gm[k] = d < D ? a.A[dir][c * D + d] : (R)0;
      gsum += gm[k];
    }
    const R gmean = warp_sum<R>(gsum) / (R)D;
    // selected term of every minimum: 0 own, 1 from d-1, 2 from d+1, 3 P2
    int sel[NV];
    R own[NV], to_prev[NV], to_next[NV], s3 = 0;
#pragma unroll
    for (int k = 0; k < NV; ++k)
    {
      const int d = lane + 32 * k;
      R prev, next;
      neighbours<NV>(hv, lane, k, prev, next);
      gm[k] = d < D ? gm[k] - gmean : (R)0;
      R best = hv[k];
      int s = 0;
      if (d > 0 && prev + P1 < best)
      {
        best = prev + P1;
        s = 1;
      }
      if (d < D - 1 && next + P1 < best)
      {
        best = next + P1;
        s = 2;
      }
      if (hmin + P2 < best)
        s = 3;
      sel[k] = d < D ? s : 0;
      own[k] = sel[k] == 0 ? gm[k] : (R)0;
      to_prev[k] = sel[k] == 1 ? gm[k] : (R)0; // lands on h(d-1)
      to_next[k] = sel[k] == 2 ? gm[k] : (R)0; // lands on h(d+1)
      if (sel[k] == 1 || sel[k] == 2)
        gp1 += gm[k];
      if (sel[k] == 3)
      {
        gp2 += gm[k];
        s3 += gm[k];
      }
    }
    s3 = warp_sum<R>(s3);
    R gh[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k)
    {
      // h(d) receives to_prev from d+1 and to_next from d-1
      R from_next, unused, from_prev;
      neighbours<NV>(to_prev, lane, k, unused, from_next);
      neighbours<NV>(to_next, lane, k, from_prev, unused);
      const int d = lane + 32 * k;
      R v = own[k];
      if (d + 1 < D)
        v += from_next;
      if (d > 0)
        v += from_prev;
      if (d == amin)
        v += s3;
      gh[k] = d < D ? v : (R)0;
    }
#pragma unroll
    for (int k = 0; k < NV; ++k)
    {
      if (dir != kUp)
        gu[k] += gh[k];
      if (dir != kDown)
        gd[k] += gh[k];
      if (dir != kLeft)
        gl[k] += gh[k];
      if (dir != kRight)
        gr[k] += gh[k];
    }
  }
#pragma unroll
  for (int k = 0; k < NV; ++k)
  {
    const int d = lane + 32 * k;
    if (d >= D)
      continue;
    if (has_u)
      a.A[kDown][(c - w) * D + d] += gu[k];
    if (has_d)
      a.A[kUp][(c + w) * D + d] += gd[k];
    if (has_l)
      a.A[kRight][(c - 1) * D + d] += gl[k];
    if (has_r)
      a.A[kLeft][(c + 1) * D + d] += gr[k];
#pragma unroll
    for (int dir = 0; dir < 4; ++dir)
      a.A[dir][c * D + d] = (R)0;
  }
  const double t1 = warp_sum<double>((double)gp1), t2 = warp_sum<double>((double)gp2);
  if (lane == 0)
  {
    atomicAdd(a.gP, t1);
    atomicAdd(a.gP + 1, t2);
  }
}

// adjoint of the copy-down: every parent message adds the adjoints of its
// (up to four) children's starting messages
template <class R>
__global__ void __launch_bounds__(256)
    k_msg_downsample_add(const MsgPtrsR<R> child, int cw, int ch, const MsgPtrsR<R> parent,
                         int pw, int ph, int D)
{
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)pw * ph * D)
    return;
  const int p = (int)(t / D), d = (int)(t - (long)p * D);
  const int px = p % pw, py = p / pw;
#pragma unroll
  for (int m = 0; m < 4; ++m)
  {
    R s = 0;
    for (int j = 0; j < 2; ++j)
      for (int i = 0; i < 2; ++i)
      {
        const int x = 2 * px + i, y = 2 * py + j;
        if (x < cw && y < ch)
          s += child.m[m][((size_t)y * cw + x) * D + d];
      }
    parent.m[m][(size_t)p * D + d] += s;
  }
}

// ------------------------------------------- FP64 BP forward (gradient check)
__global__ void __launch_bounds__(256) k_widen(const float *in, double *out, long n)
{
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n)
    out[t] = (double)in[t];
}

// cost_distribute (bpextract.cu:169-198) in FP64: children summed x offset
// outer, y offset inner
__global__ void __launch_bounds__(256)
    k_pyramid64(const double *fine, int fw, int fh, double *coarse, int cw, int ch, int D)
{
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)cw * ch * D)
    return;
  const int p = (int)(t / D), d = (int)(t - (long)p * D);
  const int x = p % cw, y = p / cw;
  double s = 0.0;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j)
      if (2 * x + i < fw && 2 * y + j < fh)
        s += fine[((size_t)(2 * y + j) * fw + (2 * x + i)) * D + d];
  coarse[t] = s;
}

// the reference's copy-down of the parent's messages (upsample,
// bpextract.cu:374-395), zeros at the coarsest level (bpextract.cu:87-90)
__global__ void __launch_bounds__(256)
    k_msg_inherit_all64(const MsgPtrs64 parent, int has_parent, int pw, const MsgPtrs64 child,
                        int cw, int ch, int D)
{
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)cw * ch * D)
    return;
  const int p = (int)(t / D), d = (int)(t - (long)p * D);
  const int x = p % cw, y = p / cw;
  const size_t src = ((size_t)(y >> 1) * pw + (x >> 1)) * D + d;
#pragma unroll
  for (int m = 0; m < 4; ++m)
    child.m[m][t] = has_parent ? parent.m[m][src] : 0.0;
}

// one half-sweep (bp, bpextract.cu:200-312) in FP64, a warp per cell of the
// colour, messages M updated in place
template <int D>
__global__ void __launch_bounds__(kDiffWarps * 32)
    k_bp_sweep_fwd64(const DiffBp64 a, const MsgPtrs64 M)
{
  using RM = Real<double>;
  constexpr int NV = (D + 31) / 32;
  const int lane = threadIdx.x & 31;
  const int w = a.w, h = a.h, hw = (w + 1) / 2;
  const int item = blockIdx.x * kDiffWarps + (threadIdx.x >> 5);
  if (item >= hw * h)
    return;
  const int y = item / hw;
  const int x = 2 * (item - y * hw) + ((y + a.parity) & 1);
  if (x >= w || skipped(a, x, y))
    return;
  const bool has_u = y > 0, has_d = y < h - 1, has_l = x > 0, has_r = x < w - 1;
  const size_t c = (size_t)y * w + x;
  double dat[NV], fu[NV], fd[NV], fl[NV], fr[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k)
  {
    const int d = lane + 32 * k;
    const bool in = d < D;
    dat[k] = in ? a.data[c * D + d] : 0.0;
    fu[k] = (in && has_u) ? M.m[kDown][(c - w) * D + d] : 0.0;
    fd[k] = (in && has_d) ? M.m[kUp][(c + w) * D + d] : 0.0;
    fl[k] = (in && has_l) ? M.m[kRight][(c - 1) * D + d] : 0.0;
    fr[k] = (in && has_r) ? M.m[kLeft][(c + 1) * D + d] : 0.0;
  }
  const double P1 = a.P1, P2 = a.P2;
#pragma unroll
  for (int dir = 0; dir < 4; ++dir)
  {
    double hv[NV];
    double lmin = RM::big();
#pragma unroll
    for (int k = 0; k < NV; ++k)
    {
      double v = dat[k];
      if (dir != kUp && has_u)
        v += fu[k];
      if (dir != kDown && has_d)
        v += fd[k];
      if (dir != kLeft && has_l)
        v += fl[k];
      if (dir != kRight && has_r)
        v += fr[k];
      hv[k] = (lane + 32 * k < D) ? v : RM::big();
      lmin = fmin(lmin, hv[k]);
    }
    const double hmin = warp_min<double>(lmin);
    double m[NV], msum = 0.0;
#pragma unroll
    for (int k = 0; k < NV; ++k)
    {
      const int d = lane + 32 * k;
      double prev, next;
      neighbours<NV>(hv, lane, k, prev, next);
      double v = hv[k];
      if (d > 0)
        v = fmin(v, prev + P1);
      if (d < D - 1)
        v = fmin(v, next + P1);
      m[k] = fmin(v, hmin + P2);
      if (d < D)
        msum += m[k];
    }
    const double mean = warp_sum<double>(msum) / (double)D;
#pragma unroll
    for (int k = 0; k < NV; ++k)
    {
      const int d = lane + 32 * k;
      if (d < D)
        M.m[dir][c * D + d] = m[k] - mean;
    }
  }
}

// ------------------------------------------------------ weighted upsampling
// Edge weight factor: exp(-(Ia - Ib)^2 / sigma) in FP64.
__device__ __forceinline__ double edge_exp(double a, double b, double sigma)
{
  const double diff = a - b;
  return exp(-diff * diff / sigma);
}

// weight of the edge (k-1, k) of a line of n samples: k = 0 -> 0, k = n ->
// the closing weight, else omega * exp term
struct LineW
{
  const uint8_t *img;
  size_t step_img; // image elements between consecutive samples
  const float *omega;
  size_t step;     // pixel elements between consecutive samples
  int n;
  double closing, sigma;
  __device__ double w(int k, double *expo = nullptr) const
  {
    if (k <= 0)
      return 0.0;
    if (k >= n)
      return closing;
    const double e = edge_exp((double)img[k * step_img], (double)img[(k - 1) * step_img], sigma);
    if (expo)
      *expo = e;
    return (double)omega[k * step] * e;
  }
};

// Solves (I + lam L_w) s = r along one line for two right-hand sides (FP64
// Thomas); cp is scratch of n doubles.  r and s may alias.
__device__ void thomas2(const LineW &L, double lam, const double *r0, const double *r1,
                        double *s0, double *s1, double *cp, size_t step)
{
  const int n = L.n;
  double wl = L.w(0), wr = L.w(1);
  double den = 1.0 + lam * (wl + wr);
  double c = -lam * wr / den;
  double d0 = r0[0] / den, d1 = r1[0] / den;
  cp[0] = c;
  s0[0] = d0;
  s1[0] = d1;
  for (int k = 1; k < n; ++k)
  {
    wl = wr;
    wr = L.w(k + 1);
    const double a = -lam * wl;
    den = 1.0 + lam * (wl + wr) - a * c;
    c = -lam * wr / den;
    d0 = (r0[k * step] - a * d0) / den;
    d1 = (r1[k * step] - a * d1) / den;
    cp[k * step] = c;
    s0[k * step] = d0;
    s1[k * step] = d1;
  }
  for (int k = n - 2; k >= 0; --k)
  {
    s0[k * step] -= cp[k * step] * s0[(k + 1) * step];
    s1[k * step] -= cp[k * step] * s1[(k + 1) * step];
  }
}

// row pass: one thread per row
__global__ void k_upw_rows_fwd(DiffUp u)
{
  const int y = blockIdx.x * blockDim.x + threadIdx.x;
  if (y >= u.H)
    return;
  const size_t o = (size_t)y * u.W;
  LineW L{u.img + (size_t)y * u.pitch, 1, u.omega + o, 1, u.W, u.row_closing, u.sigma};
  for (int x = 0; x < u.W; ++x)
  {
    const double d = u.sparse[o + x];
    u.sd[o + x] = d;
    u.si[o + x] = d > 0.0 ? 1.0 : 0.0;
  }
  thomas2(L, u.lam, u.sd + o, u.si + o, u.sd + o, u.si + o, u.cp + o, 1);
}

// column pass: one thread per column (coalesced across threads)
__global__ void k_upw_cols_fwd(DiffUp u)
{
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= u.W)
    return;
  LineW L{u.img + x, u.pitch, u.omega + x, (size_t)u.W, u.H, u.col_closing, u.sigma};
  thomas2(L, u.lam, u.sd + x, u.si + x, u.td + x, u.ti + x, u.cp + x, (size_t)u.W);
  for (int y = 0; y < u.H; ++y)
  {
    const size_t o = (size_t)y * u.W + x;
    u.dense[o] = (float)(u.td[o] / u.ti[o]);
  }
}

// column adjoint: u = B^-1 g_t, g_omega from the column edges
__global__ void k_upw_cols_bwd(DiffUp u)
{
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= u.W)
    return;
  const size_t W = u.W;
  for (int y = 0; y < u.H; ++y)
  {
    const size_t o = (size_t)y * W + x;
    const double g = u.g_dense[o], ti = u.ti[o];
    u.ud[o] = g / ti;
    u.ui[o] = -g * u.td[o] / (ti * ti);
  }
  LineW L{u.img + x, u.pitch, u.omega + x, W, u.H, u.col_closing, u.sigma};
  thomas2(L, u.lam, u.ud + x, u.ui + x, u.ud + x, u.ui + x, u.cp + x, W);
  for (int y = 1; y < u.H; ++y)
  {
    const size_t o = (size_t)y * W + x, p = o - W;
    double e = 0.0;
    L.w(y, &e);
    const double gw = -u.lam * ((u.ud[o] - u.ud[p]) * (u.td[o] - u.td[p]) +
                                (u.ui[o] - u.ui[p]) * (u.ti[o] - u.ti[p]));
    u.g_omega[o] = (float)(gw * e);
  }
  u.g_omega[x] = 0.0f;
}

// row adjoint: v = A^-1 u, g_sparse = v_d, g_omega += row edges
__global__ void k_upw_rows_bwd(DiffUp u)
{
  const int y = blockIdx.x * blockDim.x + threadIdx.x;
  if (y >= u.H)
    return;
  const size_t o = (size_t)y * u.W;
  LineW L{u.img + (size_t)y * u.pitch, 1, u.omega + o, 1, u.W, u.row_closing, u.sigma};
  thomas2(L, u.lam, u.ud + o, u.ui + o, u.ud + o, u.ui + o, u.cp + o, 1);
  for (int x = 0; x < u.W; ++x)
  {
    u.g_sparse[o + x] = (float)u.ud[o + x];
    if (x == 0)
      continue;
    double e = 0.0;
    L.w(x, &e);
    const size_t q = o + x, p = q - 1;
    const double gw = -u.lam * ((u.ud[q] - u.ud[p]) * (u.sd[q] - u.sd[p]) +
                                (u.ui[q] - u.ui[p]) * (u.si[q] - u.si[p]));
    u.g_omega[q] += (float)(gw * e);
  }
}

// ------------------------------------------------------------ fusion adjoint
struct Dual
{
  double v, g;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.g + b.g}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.g - b.g}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b)
{
  return {a.v * b.v, a.g * b.v + a.v * b.g};
}
__device__ __forceinline__ Dual operator/(Dual a, Dual b)
{
  const double q = a.v / b.v;
  return {q, (a.g - q * b.g) / b.v};
}
__device__ __forceinline__ Dual cst(double v) { return {v, 0.0}; }
__device__ __forceinline__ Dual dexp(Dual a)
{
  const double e = exp(a.v);
  return {e, e * a.g};
}
__device__ __forceinline__ Dual dsqrt(Dual a)
{
  const double s = sqrt(a.v);
  return {s, a.g / (2.0 * s)};
}

// d(fused depth)/d(upsampled depth) times the incoming gradient, with the
// prior of the pixel (table and transformed seeds of the forward fusion)
__global__ void __launch_bounds__(256) k_fuse_bwd(DiffFuse f)
{
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)f.W * f.H)
    return;
  const Dual dep{(double)f.depth_in[idx], 1.0};
  Dual unc = dep.v * 0.2 > 0.5 ? dep * cst(0.2) : cst(0.5);
  unc = unc * unc;
  if (dep.v <= 0.0)
    unc = cst(1e9);
  const int pre = f.table[idx];
  Dual a = cst(10.0), b = cst(10.0), mu = dep, s2 = cst(2500.0);
  if (pre > 0)
  {
    const float4 s = f.seeds_in[pre];
    a = cst(s.x);
    b = cst(s.y);
    mu = cst(s.z);
    s2 = cst(s.w);
  }
  if (((dep - mu) * (dep - mu)).v > (unc + s2).v)
  {
    a = cst(10.0);
    b = cst(10.0);
    mu = dep;
    s2 = cst(2500.0);
  }
  const Dual var = unc + s2;
  const Dual new_mu = (dep * s2 + mu * unc) / var;
  const Dual dm = dep - mu;
  const Dual pdf = dexp(cst(0.0) - dm * dm / (cst(2.0) * var)) / dsqrt(cst(2.0 * M_PI) * var);
  const double ratio = a.v / (a.v + b.v);
  Dual c1 = cst(ratio) * pdf;
  Dual c2 = cst(b.v / (a.v + b.v) / 50.0);
  const Dual norm = c1 + c2;
  c1 = c1 / norm;
  c2 = c2 / norm;
  const Dual mu_p = c1 * new_mu + c2 * mu;
  f.g_depth[idx] = ratio > 0.60 ? (float)(mu_p.g * (double)f.g_fused[idx]) : 0.0f;
}

template <int D, class R>
void readout_d(const DiffBpR<R> &a, int backward, cudaStream_t s)
{
  const int cells = a.w * a.h;
  k_soft_readout<D, R><<<(cells + kDiffWarps - 1) / kDiffWarps, kDiffWarps * 32, 0, s>>>(
      a, backward);
}

template <int D, class R>
void bwd_d(const DiffBpR<R> &a, cudaStream_t s)
{
  const int items = ((a.w + 1) / 2) * a.h;
  k_bp_sweep_bwd<D, R><<<(items + kDiffWarps - 1) / kDiffWarps, kDiffWarps * 32, 0, s>>>(a);
}

template <class F>
void by_d(int d, F &&f)
{
  switch (d)
  {
  case 32: f(std::integral_constant<int, 32>()); break;
  case 48: f(std::integral_constant<int, 48>()); break;
  case 64: f(std::integral_constant<int, 64>()); break;
  case 96: f(std::integral_constant<int, 96>()); break;
  case 128: f(std::integral_constant<int, 128>()); break;
  default: break;
  }
}

} // namespace

void launch_soft_readout(const DiffBp &a, int backward, cudaStream_t s)
{
  by_d(a.D, [&](auto dc) { readout_d<decltype(dc)::value>(a, backward, s); });
}

void launch_soft_readout(const DiffBp64 &a, int backward, cudaStream_t s)
{
  by_d(a.D, [&](auto dc) { readout_d<decltype(dc)::value>(a, backward, s); });
}

void launch_bp_sweep_bwd(const DiffBp &a, cudaStream_t s)
{
  by_d(a.D, [&](auto dc) { bwd_d<decltype(dc)::value>(a, s); });
}

void launch_bp_sweep_bwd(const DiffBp64 &a, cudaStream_t s)
{
  by_d(a.D, [&](auto dc) { bwd_d<decltype(dc)::value>(a, s); });
}

namespace
{
template <class R>
void downsample_add(const MsgPtrsR<R> &child, int cw, int ch, const MsgPtrsR<R> &parent, int pw,
                    int ph, int D, cudaStream_t s)
{
  const long n = (long)pw * ph * D;
  if (n > 0)
    k_msg_downsample_add<R><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(child, cw, ch, parent,
                                                                        pw, ph, D);
}
} // namespace

void launch_msg_downsample_add(const MsgPtrs &child, int cw, int ch, const MsgPtrs &parent,
                               int pw, int ph, int D, cudaStream_t s)
{
  downsample_add(child, cw, ch, parent, pw, ph, D, s);
}

void launch_msg_downsample_add(const MsgPtrs64 &child, int cw, int ch, const MsgPtrs64 &parent,
                               int pw, int ph, int D, cudaStream_t s)
{
  downsample_add(child, cw, ch, parent, pw, ph, D, s);
}

void launch_widen(const float *in, double *out, long n, cudaStream_t s)
{
  if (n > 0)
    k_widen<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(in, out, n);
}

void launch_pyramid64(const double *fine, int fw, int fh, double *coarse, int cw, int ch, int D,
                      cudaStream_t s)
{
  const long n = (long)cw * ch * D;
  if (n > 0)
    k_pyramid64<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(fine, fw, fh, coarse, cw, ch, D);
}

void launch_msg_inherit_all64(const MsgPtrs64 *parent, int pw, const MsgPtrs64 &child, int cw,
                              int ch, int D, cudaStream_t s)
{
  const long n = (long)cw * ch * D;
  MsgPtrs64 none{};
  if (n > 0)
    k_msg_inherit_all64<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(
        parent ? *parent : none, parent ? 1 : 0, pw, child, cw, ch, D);
}

void launch_bp_sweep_fwd64(const DiffBp64 &a, const MsgPtrs64 &M, cudaStream_t s)
{
  const int items = ((a.w + 1) / 2) * a.h;
  by_d(a.D, [&](auto dc) {
    k_bp_sweep_fwd64<decltype(dc)::value>
        <<<(items + kDiffWarps - 1) / kDiffWarps, kDiffWarps * 32, 0, s>>>(a, M);
  });
}

void launch_upw_forward(const DiffUp &u, cudaStream_t s)
{
  k_upw_rows_fwd<<<(u.H + 63) / 64, 64, 0, s>>>(u);
  k_upw_cols_fwd<<<(u.W + 63) / 64, 64, 0, s>>>(u);
}

void launch_upw_backward(const DiffUp &u, cudaStream_t s)
{
  k_upw_cols_bwd<<<(u.W + 63) / 64, 64, 0, s>>>(u);
  k_upw_rows_bwd<<<(u.H + 63) / 64, 64, 0, s>>>(u);
}

void launch_fuse_bwd(const DiffFuse &f, cudaStream_t s)
{
  const long n = (long)f.W * f.H;
  if (n > 0)
    k_fuse_bwd<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(f);
}

} // namespace qm
