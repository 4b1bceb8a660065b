// Bayesian Gaussian x Beta depth fusion (fuse_transform, hole_filling,
// fuse_currentmap; depth_fusion.cu:13-213 of the reference).
//
// The previous seeds (a, b, mu, sigma^2) are moved into the current frame:
// good seeds (a >= 0.001, a/(a+b) >= 0.45) have their depth moved along their
// viewing ray by T_income<-last, sigma^2 += 0.01*depth, and they compete for
// the pixel they project to.  The reference resolves the competition with a
// compare-and-swap loop that may give up or read a stale depth, and fills
// holes first-writer-wins; here both are deterministic:
//  * z-buffer: atomicMin on the 64-bit key (depth bits << 32 | source index);
//    depths are positive floats, so the key orders by depth, then by index;
//  * hole filling reads the resolved keys: an empty pixel takes the nearest
//    (smallest key) non-empty 3x3 neighbour among the pixels that propagate
//    (x in [2, W-1), y in [2, H-1)); one pass, no chains.  It runs inside
//    the update kernel (each pixel resolves its own source, then updates).

// Index 0 is the "empty" table value, so pixel (0, 0) never propagates
// (as in the reference).  The posterior update (fuse_currentmap) runs in FP64;
// the emitted depth is mu' when the PRIOR inlier ratio a/(a+b) > 0.6, else -1.
// The update kernel leaves the keys set (its neighbours may still read them);
// the batched pipeline's row solve resets them in the stream's next dense
// frame (before its transform), the stage entry point clears its workspace.
//
// Bytes per pixel: transform 16 read + 16 written (+ 8-byte atomic); update
// 4 + 8 + 16 read (+ the 3x3 keys of an empty pixel, cached), 4 + 16
// written (+ 4 when the source table is kept).
#include "launch.h"

namespace qm
{

namespace
{

constexpr unsigned long long kEmpty = ~0ull;

// e^x for the pdf's exponent x = -dm^2 / (2 var): a pixel whose squared
// distance to its prior exceeds var has been reset to its own depth (dm =
// 0), so x lies in [-0.5, 0].  There the Taylor series of e^x to degree 14,
// evaluated by Horner's rule, is accurate to the last bits of a double (the
// first dropped term is below 0.5^15 / 15! < 3e-17); any other argument
// (NaN, inf input) takes the library exp.
__device__ __forceinline__ double exp_pdf(double x)
{
  if (!(x >= -0.5 && x <= 0.0))
    return exp(x);
  // 1 / k!, k = 14 .. 0
  constexpr double c[15] = {1.0 / 87178291200.0, 1.0 / 6227020800.0, 1.0 / 479001600.0,
                            1.0 / 39916800.0,    1.0 / 3628800.0,    1.0 / 362880.0,
                            1.0 / 40320.0,       1.0 / 5040.0,       1.0 / 720.0,
                            1.0 / 120.0,         1.0 / 24.0,         1.0 / 6.0,
                            0.5,                 1.0,                1.0};
  double r = c[0];
#pragma unroll
  for (int k = 1; k < 15; ++k)
    r = fma(r, x, c[k]);
  return r;
}

// 1/v for a positive normal v: the hardware's approximate FP64 reciprocal
// refined by two Newton-Raphson steps r <- r + r (1 - v r), each of which
// squares the relative error (about 2^-22 -> 2^-44 -> below 2^-53).
__device__ __forceinline__ double recip_pos(double v)
{
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(v));
  double e = fma(-v, r, 1.0);
  r = fma(r, e, r);
  e = fma(-v, r, 1.0);
  return fma(r, e, r);
}

// pixel idx of a W-wide image: (x, y) without an integer division (idx <
// 2^24 is exact in float; the float quotient is off by at most one row)
__device__ __forceinline__ void pixel_xy(int idx, int W, float inv_w, int &x, int &y)
{
  y = (int)((float)idx * inv_w);
  if (y * W > idx)
    --y;
  else if ((y + 1) * W <= idx)
    ++y;
  x = idx - y * W;
}

// Moves one seed into the current frame and enters it in the z-buffer.
template <class A>
__device__ __forceinline__ void transform_px(const JobDesc &J, int idx, float4 info, float inv_w)
{
  const int W = J.W, H = J.H;
  // is_badpoint (depth_fusion.cu:25-28)
  if (info.x < 0.001 || A::div(info.x, info.x + info.y) < 0.45)
    return;
  int x, y;
  pixel_xy(idx, W, inv_w, x, y);
  const Cam cam{J.fx, J.fy, J.cx, J.cy};
  const float3 dir = A::ray((float)x, (float)y, cam);
  float T[12];
#pragma unroll
  for (int k = 0; k < 12; ++k)
    T[k] = J.Tf[k];
  const float3 q = A::apply(T, A::scale(dir, info.z));
  const float nd = A::length(q);
  if (nd <= 0.5)
    return;
  info.z = nd;
  if (A::kIeee)
    info.w = (float)__dadd_rn((double)info.w, __dmul_rn((double)nd, 0.01));
  else
    info.w += nd * 0.01;
  const float2 uv = A::project(q, cam);
  const int tx = trunc_int((double)uv.x + 0.5), ty = trunc_int((double)uv.y + 0.5);
  if (tx >= W || tx < 0 || ty >= H || ty < 0)
    return;
  J.seeds_in[idx] = info;
  if (idx != 0)
  {
    const unsigned long long key =
        ((unsigned long long)__float_as_uint(nd) << 32) | (unsigned long long)(unsigned)idx;
    atomicMin(J.zkey + (size_t)ty * W + tx, key);
  }
}

// kFuseTransformPx pixels per thread, their seeds loaded before any is
// processed (the loads are the latency that bounds this pass)
template <class A>
__global__ void __launch_bounds__(kFlatThreads)
    k_fuse_transform(const __grid_constant__ Batch B)
{
  int lb;
  const JobDesc &J = job_of(B, lb);
  const int npx = J.W * J.H;
  const int base = lb * (int)blockDim.x * kFuseTransformPx + (int)threadIdx.x;
  const float inv_w = 1.0f / (float)J.W;
  float4 info[kFuseTransformPx];
#pragma unroll
  for (int u = 0; u < kFuseTransformPx; ++u)
  {
    const int idx = base + u * (int)blockDim.x;
    info[u] = idx < npx ? J.seeds_in[idx] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  }
#pragma unroll
  for (int u = 0; u < kFuseTransformPx; ++u)
  {
    const int idx = base + u * (int)blockDim.x;
    if (idx < npx)
      transform_px<A>(J, idx, info[u], inv_w);
  }
}

// hole filling (hole_filling, depth_fusion.cu:121-144): the pixel's own key,
// or for an empty pixel the smallest key of its propagating 3x3 neighbours;
// returns the source seed index (0 = none)
__device__ __forceinline__ int resolve_source(const JobDesc &J, int idx, unsigned long long key,
                                              float inv_w)
{
  const int W = J.W, H = J.H;
  if (key == kEmpty)
  {
    int x, y;
    pixel_xy(idx, W, inv_w, x, y);
    for (int i = -1; i <= 1; ++i)
      for (int jx = -1; jx <= 1; ++jx)
      {
        const int nx = x + jx, ny = y + i;
        if (nx < 2 || nx >= W - 1 || ny < 2 || ny >= H - 1)
          continue;
        const unsigned long long k = J.zkey[(size_t)ny * W + nx];
        key = k < key ? k : key;
      }
  }
  return key == kEmpty ? 0 : (int)(unsigned)(key & 0xffffffffull);
}

// fuse_currentmap (depth_fusion.cu:146-213) of one pixel in FP64, given its
// upsampled depth and its prior seed (source pre > 0) or none
__device__ __forceinline__ void update_px(const JobDesc &J, int idx, double dep, int pre,
                                          float4 s)
{
  double unc = fmax(0.5, dep * 0.2);
  unc *= unc;
  if (dep <= 0.0)
    unc = 1e9;
  if (J.table)
    J.table[idx] = pre;
  double a, b, mu, s2;
  if (pre > 0)
  {
    a = s.x;
    b = s.y;
    mu = s.z;
    s2 = s.w;
  }
  else
  {
    a = 10.0;
    b = 10.0;
    mu = dep;
    s2 = 2500.0;
  }
  if ((dep - mu) * (dep - mu) > unc + s2)
  {
    a = 10.0;
    b = 10.0;
    mu = dep;
    s2 = 2500.0;
  }
  // The reference's formulas with their denominators shared and inverted once
  // (FP64 division is the costly operation here: five of them instead of
  // the reference's term-by-term quotients; the results differ from those
  // by a few FP64 ulps).  The identities used: c1 = ratio * pdf and
  // c2 = b / (a + b) / 50 are both rescaled by (a + b) before the
  // normalisation, which cancels it; 1/(ab+1) and 1/(ab+2) come from
  // 1/((ab+1)(ab+2)); and a' = (e - f) / (f - e/f), b' = a' (1 - f) / f
  // share the denominator f^2 - e.  The inlier ratio that gates the output
  // is the exact quotient.
  // var >= 0.25, c1 + c2 > 0 and (ab + 1)(ab + 2) >= 2 for every seed the
  // pipeline produces (a, b >= 0): their reciprocals take recip_pos; the
  // inlier ratio and the Beta update keep IEEE divisions (the ratio gates
  // the output; f^2 - e may vanish)
  const double var = unc + s2;
  const double ivar = recip_pos(var);
  const double new_sq = unc * s2 * ivar;
  const double new_mu = (dep * s2 + mu * unc) * ivar;
  const double dm = dep - mu;
  const double pdf = exp_pdf(-dm * dm * (0.5 * ivar)) * rsqrt(2.0 * M_PI * var);
  const double ab = a + b;
  const double ratio = a / ab;
  double c1 = a * pdf;
  double c2 = b * (1.0 / 50.0);
  const double inorm = recip_pos(c1 + c2);
  c1 *= inorm;
  c2 *= inorm;
  const double i12 = recip_pos((ab + 1.0) * (ab + 2.0));
  const double i1 = (ab + 2.0) * i12;
  const double f = (c1 * (a + 1.0) + c2 * a) * i1;
  const double e = (c1 * ((a + 1.0) * (a + 2.0)) + c2 * (a * (a + 1.0))) * i12;
  const double mu_p = c1 * new_mu + c2 * mu;
  const double s2_p = c1 * (new_sq + new_mu * new_mu) + c2 * (s2 + mu * mu) - mu_p * mu_p;
  const double q = (e - f) / (f * f - e);
  const double a_p = q * f;
  const double b_p = q * (1.0 - f);
  J.dense[idx] = (ratio > 0.60) ? (float)mu_p : -1.0f;
  J.seeds_out[idx] = make_float4((float)a_p, (float)b_p, (float)mu_p, (float)s2_p);
}

// A block owns kFlatThreads * kFuseUpdatePx consecutive pixels and walks
// them in kFuseUpdatePx steps of one pixel per thread.  The pixel chain
// (key -> source, for an empty pixel through its neighbours' keys -> source
// seed -> FP64 update) is software-pipelined: while step j's update runs,
// step j+1's source seed and step j+2's key and depth are already in flight,
// so the dependent loads overlap the arithmetic instead of stalling it.
// Every pixel's result depends only on its own inputs and on keys this
// kernel does not write, so the order changes nothing.
__global__ void __launch_bounds__(kFlatThreads)
    k_fuse_update(const __grid_constant__ Batch B)
{
  int lb;
  const JobDesc &J = job_of(B, lb);
  const int npx = J.W * J.H;
  const int step = (int)blockDim.x;
  const int base = lb * step * kFuseUpdatePx + (int)threadIdx.x;
  const float inv_w = 1.0f / (float)J.W;
  auto pix = [&](int j) { return base + j * step; };
  // step j: depth and key (loaded two steps ahead), source and its seed
  // (one step ahead)
  float dep0 = 0.0f, dep1 = 0.0f;
  unsigned long long key1 = kEmpty;
  int pre0 = 0;
  float4 src0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  {
    const int i0 = pix(0), i1 = pix(1);
    unsigned long long key0 = kEmpty;
    if (i0 < npx)
    {
      dep0 = J.dense[i0];
      key0 = J.zkey[i0];
    }
    if (kFuseUpdatePx > 1 && i1 < npx)
    {
      dep1 = J.dense[i1];
      key1 = J.zkey[i1];
    }
    pre0 = i0 < npx ? resolve_source(J, i0, key0, inv_w) : 0;
    if (pre0 > 0)
      src0 = J.seeds_in[pre0];
  }
  for (int j = 0; j < kFuseUpdatePx; ++j)
  {
    const int i0 = pix(j), i1 = pix(j + 1), i2 = pix(j + 2);
    if (i0 >= npx)
      break; // later steps are further out
    int pre1 = 0;
    float4 src1 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (j + 1 < kFuseUpdatePx && i1 < npx)
    {
      pre1 = resolve_source(J, i1, key1, inv_w);
      if (pre1 > 0)
        src1 = J.seeds_in[pre1];
    }
    float dep2 = 0.0f;
    unsigned long long key2 = kEmpty;
    if (j + 2 < kFuseUpdatePx && i2 < npx)
    {
      dep2 = J.dense[i2];
      key2 = J.zkey[i2];
    }
    update_px(J, i0, (double)dep0, pre0, src0);
    dep0 = dep1;
    pre0 = pre1;
    src0 = src1;
    dep1 = dep2;
    key1 = key2;
  }
}

// sigma^2 of every seed (the fused variance)
__global__ void __launch_bounds__(kFlatThreads)
    k_seed_variance(const float4 *__restrict__ seeds, float *__restrict__ out, long n)
{
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    out[i] = seeds[i].w;
}

} // namespace

void launch_seed_variance(const float4 *seeds, float *out, long n, cudaStream_t s)
{
  if (n > 0)
    k_seed_variance<<<(unsigned)((n + kFlatThreads - 1) / kFlatThreads), kFlatThreads, 0, s>>>(
        seeds, out, n);
}

void launch_fuse_transform(const Batch &B, int blocks, int arith, cudaStream_t s)
{
  if (arith == QM_ARITH_IEEE)
    k_fuse_transform<ArithIeee><<<blocks, kFlatThreads, 0, s>>>(B);
  else
    k_fuse_transform<ArithRef><<<blocks, kFlatThreads, 0, s>>>(B);
}

void launch_fuse_update(const Batch &B, int blocks, cudaStream_t s)
{
  k_fuse_update<<<blocks, kFlatThreads, 0, s>>>(B);
}

} // namespace qm
