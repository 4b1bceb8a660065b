// Edge-aware depth upsampling (global_upsample, depth_upsample.cu:20-302 of
// the reference): the sparse depth d and its indicator 1[d > 0] are smoothed
// by (I + lambda*L_w)^-1 along rows, then along columns, and the output is
// S(d) / S(1[d > 0]).  L_w is the weighted 1-D Laplacian with
// w = exp(-(dI)^2 / sigma) between neighbours.
//
// Design.  The reference solves each line with a serial Thomas sweep, one
// thread per line (480 threads for the row pass of a 752x480 frame).  Here a
// WARP solves a line: the line is cut into 32 contiguous segments, one per
// lane, and every recurrence of the Thomas algorithm is turned into a
// segment-local composition plus a 5-step warp scan:
//  * pivots: c'_k = c_k / (b_k - a_k c'_{k-1}) is a Moebius map of c'_{k-1};
//    a segment composes to a 2x2 matrix product (FP64, rescaled by powers of
//    two), an exclusive warp scan of the matrices gives every lane its
//    incoming pivot, and the lane then runs its pivots in FP64;
//  * forward right-hand sides: d'_k = (r_k - a_k d'_{k-1}) / den_k is affine
//    in d'_{k-1}; segments compose (FP32) and a warp scan gives the incoming
//    value;
//  * back substitution: s_k = d'_k - c'_k s_{k+1} is affine in s_{k+1};
//    a reverse warp scan gives every lane the value after its segment.
// FP64 is used for the pivots only; the right-hand sides are FP32, as in the
// reference.  Differences from the reference's serial FP32 sweep are
// rounding-level (within 1e-5 relative; closer to the FP64 oracle).
//
// The weights are computed from the image inside the solver (the reference
// builds two weight images first, depth_upsample.cu:58-93), keeping its edge
// behaviour: the closing weight of a line is 0 when the line length is a
// multiple of 16 and exp(0) = 1 otherwise (depth_upsample.cu:26-37).  Each
// warp keeps its line in shared memory in a skewed layout (segment j of lane
// l at l*mp + j, mp odd) so that lane-parallel accesses are conflict-free.
//
// Row pass: a block holds one row per warp (blockDim.x / 32 rows, chosen at
// launch); loads and stores are coalesced along the row.  Column pass: a block
// holds a stripe of one column per warp, loaded and stored cooperatively row
// by row.
// Bytes per pixel: row pass 1 (image) + 4 (sparse) read, 8 written; column
// pass 1 + 8 read, 4 written.
#include "launch.h"

#include <atomic>

namespace qm
{

namespace
{

// per line: w (weights, then alpha), rd / ri (right-hand sides, then the
// scaled right-hand sides, the forward values and the solution), cp (pivots)
constexpr int kArrays = 4;

__host__ __device__ __forceinline__ int seg_len(int n) { return (n + 31) / 32; }
__host__ __device__ __forceinline__ int seg_pitch(int n) { return seg_len(n) | 1; }
// floats of one array of a line of n samples (+1 for the closing weight)
__host__ __device__ __forceinline__ int line_floats(int n) { return 32 * seg_pitch(n) + 1; }

struct LineBuf
{
  float *w, *rd, *ri, *cp;
  int n, m, mp;
  __device__ __forceinline__ int pos(int k) const
  {
    const int l = k / m;
    return l * mp + (k - l * m);
  }
};

__device__ __forceinline__ LineBuf line_buf(float *base, int n)
{
  LineBuf b;
  const int L = line_floats(n);
  b.w = base;
  b.rd = base + L;
  b.ri = base + 2 * L;
  b.cp = base + 3 * L;
  b.n = n;
  b.m = seg_len(n);
  b.mp = seg_pitch(n);
  return b;
}

// weight between neighbours with intensities a (current) and b (previous),
// the reference's expression
template <class A>
__device__ __forceinline__ float edge_weight(float a, float b, double sigma)
{
  const float diff = a - b;
  return A::exp((float)((double)(-diff * diff) / sigma));
}

struct Mat2
{
  double a, b, c, d; // [[a, b], [c, d]]
};

__device__ __forceinline__ Mat2 mul(const Mat2 &L, const Mat2 &R)
{
  return Mat2{L.a * R.a + L.b * R.c, L.a * R.b + L.b * R.d, L.c * R.a + L.d * R.c,
              L.c * R.b + L.d * R.d};
}

// rescale by a power of two (exact) so the largest entry is in [1, 2): the
// scale is built from the exponent field of the largest magnitude
__device__ __forceinline__ Mat2 renorm(const Mat2 &M)
{
  const double mx = fmax(fmax(fabs(M.a), fabs(M.b)), fmax(fabs(M.c), fabs(M.d)));
  const int e = (__double2hiint(mx) >> 20) & 0x7ff; // mx = 1.f * 2^(e - 1023)
  if (e == 0 || e >= 2046)
    return M; // zero, subnormal, huge, inf or nan: leave as is
  const double s = __hiloint2double((2046 - e) << 20, 0); // 2^-(e - 1023)
  return Mat2{M.a * s, M.b * s, M.c * s, M.d * s};
}

__device__ __forceinline__ Mat2 shfl_up(const Mat2 &M, int off)
{
  return Mat2{__shfl_up_sync(0xffffffffu, M.a, off), __shfl_up_sync(0xffffffffu, M.b, off),
              __shfl_up_sync(0xffffffffu, M.c, off), __shfl_up_sync(0xffffffffu, M.d, off)};
}

struct Aff
{
  float g, hd, hi; // z -> g z + h (two right-hand sides)
};

// Solves the line held in `b` (w, rd, ri filled) and leaves the solution in
// rd (depth) and ri (indicator).  Whole warp.  Every element is rewritten in
// place by the lane that owns it, except w[e] (the first weight of the next
// segment), which each lane reads before the pass that overwrites w.
__device__ void solve_line(const LineBuf &b, double lam)
{
  const int lane = threadIdx.x & 31;
  const int s = min(lane * b.m, b.n);
  const int e = min(s + b.m, b.n);
  const int base = lane * b.mp; // smem position of element s
  // right weight of the segment's last element
  const float w_end = b.w[e < b.n ? b.pos(e) : 32 * b.mp];
  __syncwarp();
  // -------- pivots: segment Moebius product (apply element s first).  The
  // entries grow by at most 1 + 2*lambda per element, far inside the double
  // range for segments of <= 128 elements, so no per-step rescaling.
  Mat2 P{1.0, 0.0, 0.0, 1.0};
  for (int k = s; k < e; ++k)
  {
    const int p = base + (k - s);
    const double wl = b.w[p];
    const double wr = k + 1 < e ? b.w[p + 1] : w_end;
    const double a = -lam * wl, bb = 1.0 + lam * (wl + wr), c = -lam * wr;
    P = Mat2{c * P.c, c * P.d, bb * P.c - a * P.a, bb * P.d - a * P.b};
  }
  P = renorm(P);
  // inclusive scan (later segments on the left), then exclusive
#pragma unroll
  for (int off = 1; off < 32; off <<= 1)
  {
    const Mat2 Q = shfl_up(P, off);
    if (lane >= off)
      P = renorm(mul(P, Q));
  }
  Mat2 E = shfl_up(P, 1);
  if (lane == 0)
    E = Mat2{1.0, 0.0, 0.0, 1.0};
  const double z0 = E.b / E.d; // incoming pivot c'_{s-1} (0 for lane 0)
  // -------- pivots of the segment (FP64), forward RHS composition (FP32).
  // With the running product Q of the segment's Moebius maps, c'_k =
  // (Q.a z0 + Q.b) / D_k where D_k = Q.c z0 + Q.d, and den_k = D_k / D_{k-1},
  // so 1/den_k = D_{k-1} / D_k and c'_k = c_k / den_k.  Only the 2x2 products
  // form the serial chain; the one division per element does not feed back.
  // The forward recurrence d'_k = alpha_k d'_{k-1} + r_k / den_k keeps
  // alpha_k = -a_k / den_k (in w) and r_k / den_k (in rd, ri).
  Mat2 Q{1.0, 0.0, 0.0, 1.0};
  double Dprev = 1.0;
  Aff F{1.0f, 0.0f, 0.0f};
  for (int k = s; k < e; ++k)
  {
    const int p = base + (k - s);
    const double wl = b.w[p];
    const double wr = k + 1 < e ? b.w[p + 1] : w_end;
    const double a = -lam * wl, bb = 1.0 + lam * (wl + wr), c = -lam * wr;
    Q = Mat2{c * Q.c, c * Q.d, bb * Q.c - a * Q.a, bb * Q.d - a * Q.b};
    const double Dk = Q.c * z0 + Q.d;
    const double inv = Dprev / Dk; // 1 / den_k
    Dprev = Dk;
    b.cp[p] = (float)(c * inv);
    const float invf = (float)inv;
    const float alpha = (float)(lam * wl) * invf;
    const float qd = b.rd[p] * invf, qi = b.ri[p] * invf;
    b.w[p] = alpha;
    b.rd[p] = qd;
    b.ri[p] = qi;
    F = Aff{alpha * F.g, alpha * F.hd + qd, alpha * F.hi + qi};
  }
#pragma unroll
  for (int off = 1; off < 32; off <<= 1)
  {
    const float g = __shfl_up_sync(0xffffffffu, F.g, off);
    const float hd = __shfl_up_sync(0xffffffffu, F.hd, off);
    const float hi = __shfl_up_sync(0xffffffffu, F.hi, off);
    if (lane >= off)
      F = Aff{F.g * g, F.g * hd + F.hd, F.g * hi + F.hi};
  }
  float dprev = __shfl_up_sync(0xffffffffu, F.hd, 1);
  float iprev = __shfl_up_sync(0xffffffffu, F.hi, 1);
  if (lane == 0)
    dprev = iprev = 0.0f;
  // -------- forward RHS of the segment, back-substitution composition
  Aff G{1.0f, 0.0f, 0.0f};
  for (int k = s; k < e; ++k)
  {
    const int p = base + (k - s);
    const float alpha = b.w[p];
    dprev = alpha * dprev + b.rd[p];
    iprev = alpha * iprev + b.ri[p];
    b.rd[p] = dprev;
    b.ri[p] = iprev;
    const float cpk = b.cp[p];
    G = Aff{-G.g * cpk, G.g * dprev + G.hd, G.g * iprev + G.hi};
  }
  // suffix scan: lane l composes with the segments after it
#pragma unroll
  for (int off = 1; off < 32; off <<= 1)
  {
    const float g = __shfl_down_sync(0xffffffffu, G.g, off);
    const float hd = __shfl_down_sync(0xffffffffu, G.hd, off);
    const float hi = __shfl_down_sync(0xffffffffu, G.hi, off);
    if (lane + off < 32)
      G = Aff{G.g * g, G.g * hd + G.hd, G.g * hi + G.hi};
  }
  float zd = __shfl_down_sync(0xffffffffu, G.hd, 1);
  float zi = __shfl_down_sync(0xffffffffu, G.hi, 1);
  if (lane == 31)
    zd = zi = 0.0f;
  // -------- back substitution of the segment
  for (int k = e - 1; k >= s; --k)
  {
    const int p = base + (k - s);
    const float cpk = b.cp[p];
    zd = b.rd[p] - cpk * zd;
    zi = b.ri[p] - cpk * zi;
    b.rd[p] = zd;
    b.ri[p] = zi;
  }
  __syncwarp();
}

template <class A>
__global__ void __launch_bounds__(kMaxRowWarps * 32)
    k_row_solve(const __grid_constant__ Batch B, KParams kp, int max_n)
{
  extern __shared__ float smem[];
  int lb;
  const JobDesc &J = job_of(B, lb);
  const int W = J.W, H = J.H;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int y = lb * (int)(blockDim.x >> 5) + warp;
  if (y >= H)
    return;
  const int n = W / 16 * 16;
  LineBuf b = line_buf(smem + warp * kArrays * line_floats(max_n), n);
  const uint8_t *img = J.ref + (size_t)y * J.ref_pitch;
  const float *sp = J.sparse + (size_t)y * W;
  // the row's fusion z-buffer keys start empty for this frame's fusion (the
  // previous frame's update left them set); coalesced stores in a
  // latency-bound pass
  unsigned long long *zk = J.zkey ? J.zkey + (size_t)y * W : nullptr;
  for (int k = lane; k < n; k += 32)
  {
    const int p = b.pos(k);
    if (zk)
      zk[k] = ~0ull;
    const float I = (float)img[k];
    b.w[p] = k == 0 ? 0.0f : edge_weight<A>(I, (float)img[k - 1], kp.up_sigma);
    const float d = sp[k];
    b.rd[p] = d;
    b.ri[p] = d > 0.0f ? 1.0f : 0.0f;
  }
  if (lane == 0)
    b.w[32 * b.mp] = (n < W) ? edge_weight<A>((float)img[n], (float)img[n - 1], kp.up_sigma)
                             : (W % 16 != 0 ? 1.0f : 0.0f);
  __syncwarp();
  solve_line(b, kp.up_lambda);
  float2 *out = J.rowres + (size_t)y * W;
  for (int k = lane; k < n; k += 32)
  {
    const int p = b.pos(k);
    out[k] = make_float2(b.rd[p], b.ri[p]);
  }
}

template <class A>
__global__ void __launch_bounds__(kMaxColLines * 32)
    k_col_solve(const __grid_constant__ Batch B, KParams kp, int max_n)
{
  extern __shared__ float smem[];
  int lb;
  const JobDesc &J = job_of(B, lb);
  const int W = J.W, H = J.H;
  const int warp = threadIdx.x >> 5;
  const int lines = blockDim.x >> 5;
  const int x0 = lb * lines;
  const int n = H / 8 * 8;
  const int per_line = kArrays * line_floats(max_n);
  // cooperative stripe load: row k, column x0 + c
  for (int t = threadIdx.x; t < n * lines; t += blockDim.x)
  {
    const int k = t / lines, c = t - k * lines;
    const int x = x0 + c;
    if (x >= W)
      continue;
    LineBuf b = line_buf(smem + c * per_line, n);
    const int p = b.pos(k);
    const float2 r = J.rowres[(size_t)k * W + x];
    b.rd[p] = r.x;
    b.ri[p] = r.y;
    const float I = (float)J.ref[(size_t)k * J.ref_pitch + x];
    b.w[p] = k == 0 ? 0.0f
                    : edge_weight<A>(I, (float)J.ref[(size_t)(k - 1) * J.ref_pitch + x],
                                     kp.up_sigma);
    if (k == n - 1)
      b.w[32 * b.mp] =
          (n < H) ? edge_weight<A>((float)J.ref[(size_t)n * J.ref_pitch + x], I, kp.up_sigma)
                  : (H % 16 != 0 ? 1.0f : 0.0f);
  }
  __syncthreads();
  if (x0 + warp < W)
    solve_line(line_buf(smem + warp * per_line, n), kp.up_lambda);
  __syncthreads();
  for (int t = threadIdx.x; t < n * lines; t += blockDim.x)
  {
    const int k = t / lines, c = t - k * lines;
    const int x = x0 + c;
    if (x >= W)
      continue;
    LineBuf b = line_buf(smem + c * per_line, n);
    const int p = b.pos(k);
    J.dense[(size_t)k * W + x] = A::div(b.rd[p], b.ri[p]);
  }
}

} // namespace

size_t row_solve_smem(int max_w, int rows)
{
  return sizeof(float) * rows * kArrays * line_floats(max_w);
}
size_t col_solve_smem(int max_h, int lines)
{
  return sizeof(float) * lines * kArrays * line_floats(max_h);
}

void prepare_upsample_kernels()
{
  const int mx = kMaxBlockSmem;
  cudaFuncSetAttribute(k_row_solve<ArithRef>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_row_solve<ArithIeee>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_col_solve<ArithRef>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_col_solve<ArithIeee>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
}

namespace
{
// Lines longer than about 1000 elements need more than the default 48 KB of
// dynamic shared memory; the opt-in is a per-device function attribute, so
// the launchers set it once for every device they launch on (stage calls may
// run without an engine having been created on that device).
std::atomic<unsigned long long> g_prepared_devices{0};

void prepare_once_for_current_device()
{
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
  {
    prepare_upsample_kernels();
    return;
  }
  const unsigned long long bit = 1ull << dev;
  if (g_prepared_devices.load(std::memory_order_acquire) & bit)
    return;
  prepare_upsample_kernels();
  g_prepared_devices.fetch_or(bit, std::memory_order_acq_rel);
}
} // namespace

void launch_row_solve(const Batch &B, int blocks, KParams kp, int arith, int max_w,
                      cudaStream_t s, int rows)
{
  prepare_once_for_current_device();
  const size_t sm = row_solve_smem(max_w, rows);
  if (arith == QM_ARITH_IEEE)
    k_row_solve<ArithIeee><<<blocks, rows * 32, sm, s>>>(B, kp, max_w);
  else
    k_row_solve<ArithRef><<<blocks, rows * 32, sm, s>>>(B, kp, max_w);
}

void launch_col_solve(const Batch &B, int blocks, KParams kp, int arith, int max_h,
                      cudaStream_t s, int lines)
{
  prepare_once_for_current_device();
  const size_t sm = col_solve_smem(max_h, lines);
  if (arith == QM_ARITH_IEEE)
    k_col_solve<ArithIeee><<<blocks, lines * 32, sm, s>>>(B, kp, max_h);
  else
    k_col_solve<ArithRef><<<blocks, lines * 32, sm, s>>>(B, kp, max_h);
}

} // namespace qm
