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

// Dynamic shared memory of both solvers, addressed by byte offsets from this
// one symbol so that every access is a shared-memory access.  Block layout:
// the 256-entry weight table, then one line after the other.
extern __shared__ __align__(16) unsigned char g_smem[];

constexpr int kTableBytes = 256 * sizeof(float);

__device__ __forceinline__ float *smf(int byte_off)
{
  return reinterpret_cast<float *>(g_smem + byte_off);
}

__host__ __device__ __forceinline__ int seg_len(int n) { return (n + 31) / 32; }
// float pitch of a lane's segment (odd: lane-parallel accesses hit 32
// different banks)
__host__ __device__ __forceinline__ int seg_pitch(int n) { return seg_len(n) | 1; }
// byte pitch of a lane's segment of image bytes: 4 x odd, so that the 32
// lanes' bytes at the same step lie in 32 different bank words
__host__ __device__ __forceinline__ int seg_bytes(int n) { return (((seg_len(n) + 3) / 4) | 1) * 4; }
__host__ __device__ __forceinline__ int farray_bytes(int n)
{
  return (32 * seg_pitch(n) * (int)sizeof(float) + 15) & ~15;
}
// bytes of one line: three float arrays (right-hand sides, pivots) and the
// image bytes
__host__ __device__ __forceinline__ int line_bytes(int n)
{
  return 3 * farray_bytes(n) + ((32 * seg_bytes(n) + 15) & ~15);
}

// One line of n samples in shared memory, as byte offsets: rd / ri hold the
// two right-hand sides (the sparse depth and its indicator), later their
// forward values and the solution; cp the reciprocal pivots, later the
// eliminated super-diagonal; img the line's image bytes, from which every
// pass looks the weights up again.
struct Line
{
  int rd, ri, cp, img;
  int n, m, mp, bp;
  float w_close; // weight between samples n - 1 and n (the closing weight)
  __device__ __forceinline__ int fpos(int k) const
  {
    const int l = k / m;
    return l * mp + (k - l * m);
  }
  __device__ __forceinline__ int bpos(int k) const
  {
    const int l = k / m;
    return l * bp + (k - l * m);
  }
  __device__ __forceinline__ float &RD(int p) const { return smf(rd)[p]; }
  __device__ __forceinline__ float &RI(int p) const { return smf(ri)[p]; }
  __device__ __forceinline__ float &CP(int p) const { return smf(cp)[p]; }
  __device__ __forceinline__ int I(int k) const { return g_smem[img + bpos(k)]; }
};

__device__ __forceinline__ Line line_at(int base, int n, float w_close)
{
  Line L;
  const int fb = farray_bytes(n);
  L.rd = base;
  L.ri = base + fb;
  L.cp = base + 2 * fb;
  L.img = base + 3 * fb;
  L.n = n;
  L.m = seg_len(n);
  L.mp = seg_pitch(n);
  L.bp = seg_bytes(n);
  L.w_close = w_close;
  return L;
}

// weight between neighbours with intensities a (current) and b (previous),
// the reference's expression
template <class A>
__device__ __forceinline__ float edge_weight(float a, float b, double sigma)
{
  const float diff = a - b;
  return A::exp((float)((double)(-diff * diff) / sigma));
}

// The weight depends only on |I_k - I_{k-1}| (integers 0..255): a block
// tabulates edge_weight for every difference once and the passes look it
// up (the same values the expression gives pixel by pixel).
template <class A>
__device__ __forceinline__ void build_weight_table(double sigma)
{
  for (int t = threadIdx.x; t < 256; t += blockDim.x)
    smf(0)[t] = edge_weight<A>((float)t, 0.0f, sigma);
}

// weight between samples k - 1 and k of the line (k in 1 .. n - 1), given
// their intensities
__device__ __forceinline__ float table_weight(int a, int b)
{
  return smf(0)[a > b ? a - b : b - a];
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

// Walks the weights of segment [s, e): calls f(k, wl, wr) with the weights
// to the left and right of sample k.  w_0 = 0, w_n = the closing weight,
// every other from the table.
template <class Fn>
__device__ __forceinline__ void walk_weights(const Line &L, int s, int e, Fn &&f)
{
  if (s >= e)
    return;
  int Ik = L.I(s);
  float wl = s == 0 ? 0.0f : table_weight(Ik, L.I(s - 1));
  for (int k = s; k < e; ++k)
  {
    float wr;
    int In = 0;
    if (k + 1 < L.n)
    {
      In = L.I(k + 1);
      wr = table_weight(In, Ik);
    }
    else
      wr = L.w_close;
    f(k, wl, wr);
    wl = wr;
    Ik = In;
  }
}

// Solves the line (rd, ri and img filled) and leaves the solution in rd
// (depth) and ri (indicator).  Whole warp; every float element is rewritten
// in place by the lane that owns it (the image bytes are read-only).
__device__ __forceinline__ void solve_line(const Line &L, double lam)
{
  const int lane = threadIdx.x & 31;
  const int s = min(lane * L.m, L.n);
  const int e = min(s + L.m, L.n);
  const int base = lane * L.mp; // float position of element s
  // -------- pivots: segment Moebius product (apply element s first).  The
  // entries grow by at most 1 + 2*lambda per element, far inside the double
  // range for segments of <= 128 elements, so no per-step rescaling.
  Mat2 P{1.0, 0.0, 0.0, 1.0};
  walk_weights(L, s, e, [&](int, float wl_f, float wr_f) {
    const double wl = wl_f, wr = wr_f;
    const double a = -lam * wl, bb = 1.0 + lam * (wl + wr), c = -lam * wr;
    P = Mat2{c * P.c, c * P.d, bb * P.c - a * P.a, bb * P.d - a * P.b};
  });
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
  // -------- reciprocal pivots of the segment (FP64), forward RHS
  // composition (FP32).  With the running product Q of the segment's Moebius
  // maps, D_k = Q.c z0 + Q.d and den_k = D_k / D_{k-1}, so 1/den_k =
  // D_{k-1} / D_k: only the 2x2 products form the serial chain.  The forward
  // recurrence d'_k = alpha_k d'_{k-1} + r_k / den_k has alpha_k = -a_k /
  // den_k; 1/den_k is kept (as float) for the next pass.
  Mat2 Q{1.0, 0.0, 0.0, 1.0};
  double Dprev = 1.0;
  Aff F{1.0f, 0.0f, 0.0f};
  walk_weights(L, s, e, [&](int k, float wl_f, float wr_f) {
    const int p = base + (k - s);
    const double wl = wl_f, wr = wr_f;
    const double a = -lam * wl, bb = 1.0 + lam * (wl + wr), c = -lam * wr;
    Q = Mat2{c * Q.c, c * Q.d, bb * Q.c - a * Q.a, bb * Q.d - a * Q.b};
    const double Dk = Q.c * z0 + Q.d;
    const float invf = (float)(Dprev / Dk);
    Dprev = Dk;
    L.CP(p) = invf;
    const float alpha = (float)(lam * wl) * invf;
    F = Aff{alpha * F.g, alpha * F.hd + L.RD(p) * invf, alpha * F.hi + L.RI(p) * invf};
  });
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
  // -------- forward values of the segment, eliminated super-diagonal
  // c'_k = c_k / den_k, back-substitution composition
  Aff G{1.0f, 0.0f, 0.0f};
  walk_weights(L, s, e, [&](int k, float wl_f, float wr_f) {
    const int p = base + (k - s);
    const float invf = L.CP(p);
    const float alpha = (float)(lam * (double)wl_f) * invf;
    const float cpk = (float)(-lam * (double)wr_f * (double)invf);
    dprev = alpha * dprev + L.RD(p) * invf;
    iprev = alpha * iprev + L.RI(p) * invf;
    L.RD(p) = dprev;
    L.RI(p) = iprev;
    L.CP(p) = cpk;
    G = Aff{-G.g * cpk, G.g * dprev + G.hd, G.g * iprev + G.hi};
  });
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
    const float cpk = L.CP(p);
    zd = L.RD(p) - cpk * zd;
    zi = L.RI(p) - cpk * zi;
    L.RD(p) = zd;
    L.RI(p) = zi;
  }
  __syncwarp();
}

template <class A>
__global__ void __launch_bounds__(kMaxRowWarps * 32)
    k_row_solve(const __grid_constant__ Batch B, KParams kp, int max_n)
{
  int lb;
  const JobDesc &J = job_of(B, lb);
  build_weight_table<A>(kp.up_sigma);
  __syncthreads();
  const int W = J.W, H = J.H;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int y = lb * (int)(blockDim.x >> 5) + warp;
  if (y >= H)
    return;
  const int n = W / 16 * 16;
  const uint8_t *img = J.ref + (size_t)y * J.ref_pitch;
  const float w_close = (n < W) ? edge_weight<A>((float)img[n], (float)img[n - 1], kp.up_sigma)
                                : (W % 16 != 0 ? 1.0f : 0.0f);
  const Line L = line_at(kTableBytes + warp * line_bytes(max_n), n, w_close);
  const float *sp = J.sparse + (size_t)y * W;
  // the row's fusion z-buffer keys start empty for this frame's fusion (the
  // previous frame's update left them set); coalesced stores in a
  // latency-bound pass
  unsigned long long *zk = J.zkey ? J.zkey + (size_t)y * W : nullptr;
  for (int k = lane; k < n; k += 32)
  {
    const int p = L.fpos(k);
    if (zk)
      zk[k] = ~0ull;
    g_smem[L.img + L.bpos(k)] = img[k];
    const float d = sp[k];
    L.RD(p) = d;
    L.RI(p) = d > 0.0f ? 1.0f : 0.0f;
  }
  __syncwarp();
  solve_line(L, kp.up_lambda);
  float2 *out = J.rowres + (size_t)y * W;
  for (int k = lane; k < n; k += 32)
  {
    const int p = L.fpos(k);
    out[k] = make_float2(L.RD(p), L.RI(p));
  }
}

template <class A>
__global__ void __launch_bounds__(kMaxColLines * 32)
    k_col_solve(const __grid_constant__ Batch B, KParams kp, int max_n)
{
  int lb;
  const JobDesc &J = job_of(B, lb);
  build_weight_table<A>(kp.up_sigma);
  const int W = J.W, H = J.H;
  const int warp = threadIdx.x >> 5;
  const int lines = blockDim.x >> 5;
  const int x0 = lb * lines;
  const int n = H / 8 * 8;
  const int per_line = line_bytes(max_n);
  // cooperative stripe load: row k, column x0 + c
  for (int t = threadIdx.x; t < n * lines; t += blockDim.x)
  {
    const int k = t / lines, c = t - k * lines;
    const int x = x0 + c;
    if (x >= W)
      continue;
    const Line L = line_at(kTableBytes + c * per_line, n, 0.0f);
    const int p = L.fpos(k);
    const float2 r = J.rowres[(size_t)k * W + x];
    L.RD(p) = r.x;
    L.RI(p) = r.y;
    g_smem[L.img + L.bpos(k)] = J.ref[(size_t)k * J.ref_pitch + x];
  }
  __syncthreads();
  const int x = x0 + warp;
  if (x < W)
  {
    const float w_close =
        (n < H) ? edge_weight<A>((float)J.ref[(size_t)n * J.ref_pitch + x],
                                 (float)J.ref[(size_t)(n - 1) * J.ref_pitch + x], kp.up_sigma)
                : (H % 16 != 0 ? 1.0f : 0.0f);
    solve_line(line_at(kTableBytes + warp * per_line, n, w_close), kp.up_lambda);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < n * lines; t += blockDim.x)
  {
    const int k = t / lines, c = t - k * lines;
    const int xc = x0 + c;
    if (xc >= W)
      continue;
    const Line L = line_at(kTableBytes + c * per_line, n, 0.0f);
    const int p = L.fpos(k);
    J.dense[(size_t)k * W + xc] = A::div(L.RD(p), L.RI(p));
  }
}

} // namespace

size_t row_solve_smem(int max_w, int rows)
{
  return (size_t)kTableBytes + (size_t)rows * line_bytes(max_w);
}
size_t col_solve_smem(int max_h, int lines)
{
  return (size_t)kTableBytes + (size_t)lines * line_bytes(max_h);
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
