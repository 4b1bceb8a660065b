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

// Segment of a lane: m samples, m a multiple of 4 so that a segment is
// walked in chunks of four (one 16-byte shared load or store per array and
// chunk).  Line lengths are multiples of 8, so every segment is whole chunks.
__host__ __device__ __forceinline__ int seg_len(int n) { return ((n + 31) / 32 + 3) & ~3; }
// pitch of a lane's segment, in floats for the float arrays and in bytes for
// the image bytes: 4 x odd >= m, so that the eight lanes of a 16-byte access
// phase (and the 32 lanes of a 4-byte one) hit different banks
__host__ __device__ __forceinline__ int seg_pitch(int n) { return 4 * ((seg_len(n) / 4) | 1); }
__host__ __device__ __forceinline__ int farray_bytes(int n)
{
  return 32 * seg_pitch(n) * (int)sizeof(float);
}
// bytes of one line: three float arrays (right-hand sides, pivots) and the
// image bytes
__host__ __device__ __forceinline__ int line_bytes(int n)
{
  return 3 * farray_bytes(n) + 32 * seg_pitch(n);
}

// One line of n samples in shared memory, as byte offsets: rd / ri hold the
// two right-hand sides (the sparse depth and its indicator), later their
// forward values and the solution; cp the reciprocal pivots, later the
// eliminated super-diagonal; img the line's image bytes, from which every
// pass looks the weights up again.  Sample k of lane l = k / m sits at
// l * mp + k % m in each array.
struct Line
{
  int rd, ri, cp, img;
  int n, m, mp;
  unsigned m_inv; // ceil(2^32 / m): k / m = umulhi(k, m_inv) for 0 <= k < 2^20
  float w_close;  // weight between samples n - 1 and n (the closing weight)
  __device__ __forceinline__ int pos(int k) const
  {
    // with m_inv = (2^32 + e) / m, 0 <= e < m, umulhi gives floor(k/m + k e /
    // (m 2^32)), exact while k e < 2^32 (k < 2^20 here, m <= 132)
    const int l = (int)__umulhi((unsigned)k, m_inv);
    return l * mp + (k - l * m);
  }
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
  L.m_inv = 0xffffffffu / (unsigned)L.m + 1u;
  L.w_close = w_close;
  return L;
}

__device__ __forceinline__ float4 ld4(int arr, int p)
{
  return *reinterpret_cast<const float4 *>(g_smem + arr + 4 * p);
}
__device__ __forceinline__ void st4(int arr, int p, float4 v)
{
  *reinterpret_cast<float4 *>(g_smem + arr + 4 * p) = v;
}
__device__ __forceinline__ float f4(const float4 &v, int t)
{
  return t == 0 ? v.x : t == 1 ? v.y : t == 2 ? v.z : v.w;
}
__device__ __forceinline__ void set4(float4 &v, int t, float x)
{
  if (t == 0)
    v.x = x;
  else if (t == 1)
    v.y = x;
  else if (t == 2)
    v.z = x;
  else
    v.w = x;
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

// weight between samples with intensities a and b
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

// 1 / v for a positive normal v: the hardware's approximate FP64 reciprocal
// refined by two Newton-Raphson steps r <- r + r (1 - v r), each of which
// squares the relative error (about 2^-22 -> 2^-44 -> below 2^-53)
__device__ __forceinline__ double recip_pos(double v)
{
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(v));
  double e = fma(-v, r, 1.0);
  r = fma(r, e, r);
  e = fma(-v, r, 1.0);
  return fma(r, e, r);
}

struct Aff
{
  float g, hd, hi; // z -> g z + h (two right-hand sides)
};

// Walks the lane's segment [s, e) chunk by chunk (s = lane * m, element s at
// position base = lane * mp): calls f(k, wl[4], wr[4]) with the weights left
// and right of samples k .. k + 3.  w_0 = 0, w_n = the closing weight, every
// other from the table.  The image bytes of the next chunk are fetched
// before the current chunk is processed.  A segment that does not end the
// line holds all m samples, so the sample after it is the next lane's first
// (position base + mp) and the one before a segment with s > 0 is the
// previous lane's last (position base - mp + m - 1).
template <class Fn>
__device__ __forceinline__ void walk_chunks(const Line &L, int s, int e, int base, Fn &&f)
{
  if (s >= e)
    return;
  const unsigned *wimg = reinterpret_cast<const unsigned *>(g_smem + L.img + base);
  unsigned word = wimg[0];
  float w0 =
      s == 0 ? 0.0f : table_weight((int)(word & 0xffu), g_smem[L.img + base - L.mp + L.m - 1]);
  for (int k = s; k < e; k += 4)
  {
    const unsigned next = k + 4 < e     ? wimg[(k + 4 - s) >> 2]
                          : k + 4 < L.n ? *reinterpret_cast<const unsigned *>(
                                              g_smem + L.img + base + L.mp)
                                        : 0u;
    float wl[4], wr[4];
    int I[5];
#pragma unroll
    for (int t = 0; t < 4; ++t)
      I[t] = (int)((word >> (8 * t)) & 0xffu);
    I[4] = (int)(next & 0xffu);
#pragma unroll
    for (int t = 0; t < 4; ++t)
    {
      wl[t] = w0;
      w0 = k + t + 1 == L.n ? L.w_close : table_weight(I[t + 1], I[t]);
      wr[t] = w0;
    }
    f(k, wl, wr);
    word = next;
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
  walk_chunks(L, s, e, base, [&](int, const float(&wl)[4], const float(&wr)[4]) {
#pragma unroll
    for (int t = 0; t < 4; ++t)
    {
      const double a = -lam * (double)wl[t], c = -lam * (double)wr[t];
      const double bb = 1.0 + lam * ((double)wl[t] + (double)wr[t]);
      P = Mat2{c * P.c, c * P.d, bb * P.c - a * P.a, bb * P.d - a * P.b};
    }
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
  walk_chunks(L, s, e, base, [&](int k, const float(&wl)[4], const float(&wr)[4]) {
    const int p = base + (k - s);
    const float4 rd = ld4(L.rd, p), ri = ld4(L.ri, p);
    float4 inv4;
#pragma unroll
    for (int t = 0; t < 4; ++t)
    {
      const double a = -lam * (double)wl[t], c = -lam * (double)wr[t];
      const double bb = 1.0 + lam * ((double)wl[t] + (double)wr[t]);
      Q = Mat2{c * Q.c, c * Q.d, bb * Q.c - a * Q.a, bb * Q.d - a * Q.b};
      const double Dk = Q.c * z0 + Q.d;
      const float invf = (float)(Dprev * recip_pos(Dk));
      Dprev = Dk;
      set4(inv4, t, invf);
      const float alpha = (float)(lam * (double)wl[t]) * invf;
      F = Aff{alpha * F.g, alpha * F.hd + f4(rd, t) * invf, alpha * F.hi + f4(ri, t) * invf};
    }
    st4(L.cp, p, inv4);
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
  walk_chunks(L, s, e, base, [&](int k, const float(&wl)[4], const float(&wr)[4]) {
    const int p = base + (k - s);
    const float4 inv4 = ld4(L.cp, p);
    float4 rd = ld4(L.rd, p), ri = ld4(L.ri, p), cp4;
#pragma unroll
    for (int t = 0; t < 4; ++t)
    {
      const float invf = f4(inv4, t);
      const float alpha = (float)(lam * (double)wl[t]) * invf;
      const float cpk = (float)(-lam * (double)wr[t] * (double)invf);
      dprev = alpha * dprev + f4(rd, t) * invf;
      iprev = alpha * iprev + f4(ri, t) * invf;
      set4(rd, t, dprev);
      set4(ri, t, iprev);
      set4(cp4, t, cpk);
      G = Aff{-G.g * cpk, G.g * dprev + G.hd, G.g * iprev + G.hi};
    }
    st4(L.rd, p, rd);
    st4(L.ri, p, ri);
    st4(L.cp, p, cp4);
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
  // -------- back substitution of the segment, chunk by chunk from the end
  for (int k = e - 4; k >= s; k -= 4)
  {
    const int p = base + (k - s);
    const float4 cp4 = ld4(L.cp, p);
    float4 rd = ld4(L.rd, p), ri = ld4(L.ri, p);
#pragma unroll
    for (int t = 3; t >= 0; --t)
    {
      zd = f4(rd, t) - f4(cp4, t) * zd;
      zi = f4(ri, t) - f4(cp4, t) * zi;
      set4(rd, t, zd);
      set4(ri, t, zi);
    }
    st4(L.rd, p, rd);
    st4(L.ri, p, ri);
  }
  __syncwarp();
}

// elements one lane loads before it stores them (global loads in flight)
constexpr int kLoadBatch = 8;

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
  for (int k0 = lane; k0 < n; k0 += 32 * kLoadBatch)
  {
    uint8_t iv[kLoadBatch];
    float dv[kLoadBatch];
#pragma unroll
    for (int u = 0; u < kLoadBatch; ++u)
    {
      const int k = k0 + 32 * u;
      iv[u] = k < n ? img[k] : 0;
      dv[u] = k < n ? sp[k] : 0.0f;
    }
#pragma unroll
    for (int u = 0; u < kLoadBatch; ++u)
    {
      const int k = k0 + 32 * u;
      if (k >= n)
        break;
      if (zk)
        zk[k] = ~0ull;
      const int p = L.pos(k);
      g_smem[L.img + p] = iv[u];
      smf(L.rd)[p] = dv[u];
      smf(L.ri)[p] = dv[u] > 0.0f ? 1.0f : 0.0f;
    }
  }
  __syncwarp();
  solve_line(L, kp.up_lambda);
  float2 *out = J.rowres + (size_t)y * W;
  for (int k = lane; k < n; k += 32)
  {
    const int p = L.pos(k);
    out[k] = make_float2(smf(L.rd)[p], smf(L.ri)[p]);
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
  // cooperative stripe load: thread t owns column x0 + t % lines and rows
  // t / lines + 32 j (blockDim.x = 32 lines); a batch of loads per thread in
  // flight before their shared-memory stores
  const int kt = (int)threadIdx.x / lines, c = (int)threadIdx.x - kt * lines;
  const int xt = x0 + c;
  const Line Lt = line_at(kTableBytes + c * per_line, n, 0.0f);
  if (xt < W)
  {
    const float2 *rsrc = J.rowres + (size_t)kt * W + xt;
    const uint8_t *isrc = J.ref + (size_t)kt * J.ref_pitch + xt;
    const size_t rstep = (size_t)32 * W, istep = (size_t)32 * J.ref_pitch;
    for (int k0 = kt; k0 < n; k0 += 32 * kLoadBatch)
    {
      float2 rv[kLoadBatch];
      uint8_t iv[kLoadBatch];
#pragma unroll
      for (int u = 0; u < kLoadBatch; ++u)
      {
        const bool in = k0 + 32 * u < n;
        rv[u] = in ? rsrc[u * rstep] : make_float2(0.0f, 0.0f);
        iv[u] = in ? isrc[u * istep] : 0;
      }
#pragma unroll
      for (int u = 0; u < kLoadBatch; ++u)
      {
        const int k = k0 + 32 * u;
        if (k >= n)
          break;
        const int p = Lt.pos(k);
        smf(Lt.rd)[p] = rv[u].x;
        smf(Lt.ri)[p] = rv[u].y;
        g_smem[Lt.img + p] = iv[u];
      }
      rsrc += kLoadBatch * rstep;
      isrc += kLoadBatch * istep;
    }
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
  if (xt < W)
  {
    float *dst = J.dense + (size_t)kt * W + xt;
    for (int k = kt; k < n; k += 32, dst += (size_t)32 * W)
    {
      const int p = Lt.pos(k);
      *dst = A::div(smf(Lt.rd)[p], smf(Lt.ri)[p]);
    }
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
