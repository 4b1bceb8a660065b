// Edge-aware depth upsampling (global_upsample, depth_upsample.cu:20-302 of
// the reference): the sparse depth d and its indicator 1[d > 0] are smoothed
// by (I + lambda*L_w)^-1 along rows, then along columns, and the output is
// S(d) / S(1[d > 0]).  L_w is the weighted 1-D Laplacian with
// w = exp(-(dI)^2 / sigma) between neighbours.
//
// Differences from the reference, by design:
//  * the forward elimination (pivots and eliminated right-hand sides) runs in
//    FP64, the back substitution too; results are rounded to float between
//    the row and column passes and at the end (the reference is FP32
//    throughout with approximate divisions).  Agreement with the reference is
//    within 1e-5 relative; with the FP64 oracle within a few float ulps.
//  * the forward coefficients are stored transposed ([x][y] for the row pass)
//    so that consecutive threads (rows) store consecutive addresses.
// The weight images keep the reference's edge behaviour: the weight grid
// spans ceil(W/16)*16 x ceil(H/16)*16 threads, so row_w(W, .) / col_w(., H)
// are exp(0) = 1 when W / H are not multiples of 16, 0 otherwise
// (depth_upsample.cu:26-37, 64-93).
//
// Bytes per pixel: weights 1 read (u8) + 8 written; row pass 4+8 read,
// 24 written and read back, 8 written; column pass 8+4 read, 24+24, 4 written.
#include "launch.h"

namespace qm
{

namespace
{

template <class A>
__global__ void __launch_bounds__(kFlatThreads)
    k_weights(const __grid_constant__ Batch B, KParams kp)
{
  int lb;
  const JobDesc &J = job_of(B, lb);
  const int W = J.W, H = J.H;
  const long t = (long)lb * blockDim.x + threadIdx.x;
  if (t >= (long)(W + 1) * (H + 1))
    return;
  const int x = (int)(t % (W + 1)), y = (int)(t / (W + 1));
  const int gw = (W + 15) / 16 * 16, gh = (H + 15) / 16 * 16;
  auto I = [&](int xx, int yy) {
    xx = min(max(xx, 0), W - 1);
    yy = min(max(yy, 0), H - 1);
    return (float)J.ref[(size_t)yy * J.ref_pitch + xx];
  };
  if (y < H)
  {
    float w = 0.0f;
    if (x >= 1 && x < gw)
    {
      const float diff = I(x, y) - I(x - 1, y);
      w = A::exp((float)((double)(-diff * diff) / kp.up_sigma));
    }
    J.row_w[(size_t)y * (W + 1) + x] = w;
  }
  if (x < W)
  {
    float w = 0.0f;
    if (y >= 1 && y < gh)
    {
      const float diff = I(x, y) - I(x, y - 1);
      w = A::exp((float)((double)(-diff * diff) / kp.up_sigma));
    }
    J.col_w[(size_t)y * W + x] = w;
  }
}

// One thread per row.  Row pass of global_upsample (smooth_row,
// depth_upsample.cu:94-197) over the first W/16*16 samples.
__global__ void __launch_bounds__(kLineThreads)
    k_row_solve(const __grid_constant__ Batch B, KParams kp)
{
  int lb;
  const JobDesc &J = job_of(B, lb);
  const int W = J.W, H = J.H;
  const int y = lb * blockDim.x + threadIdx.x;
  if (y >= H)
    return;
  const int n = W / 16 * 16;
  if (n == 0)
    return;
  const double lam = kp.up_lambda;
  const float *wrow = J.row_w + (size_t)y * (W + 1);
  const float *sp = J.sparse + (size_t)y * W;
  double *tc = J.tmp, *td = J.tmp + (size_t)W * H, *ti = J.tmp + 2 * (size_t)W * H;
  double fc = 0.0, fd = 0.0, fi = 0.0;
  double wl = 0.0;
  for (int x = 0; x < n; ++x)
  {
    const double wr = (double)wrow[x + 1];
    const float dep = sp[x];
    const double ind = dep > 0.0f ? 1.0 : 0.0;
    const double a = -lam * wl;
    const double b = 1.0 + lam * (wl + wr);
    const double c = -lam * wr;
    const double inv = 1.0 / (b - fc * a);
    fc = c * inv;
    fd = ((double)dep - fd * a) * inv;
    fi = (ind - fi * a) * inv;
    const size_t o = (size_t)x * H + y;
    tc[o] = fc;
    td[o] = fd;
    ti[o] = fi;
    wl = wr;
  }
  double nd = 0.0, ni = 0.0;
  for (int x = n - 1; x >= 0; --x)
  {
    const size_t o = (size_t)x * H + y;
    const double cc = tc[o];
    nd = td[o] - cc * nd;
    ni = ti[o] - cc * ni;
    J.rowres[(size_t)y * W + x] = make_float2((float)nd, (float)ni);
  }
}

// One thread per column.  Column pass (smooth_col, depth_upsample.cu:198-302)
// over the first H/8*8 rows, writing S(d)/S(ind).
__global__ void __launch_bounds__(kLineThreads)
    k_col_solve(const __grid_constant__ Batch B, KParams kp)
{
  int lb;
  const JobDesc &J = job_of(B, lb);
  const int W = J.W, H = J.H;
  const int x = lb * blockDim.x + threadIdx.x;
  if (x >= W)
    return;
  const int n = H / 8 * 8;
  if (n == 0)
    return;
  const double lam = kp.up_lambda;
  double *tc = J.tmp, *td = J.tmp + (size_t)W * H, *ti = J.tmp + 2 * (size_t)W * H;
  double fc = 0.0, fd = 0.0, fi = 0.0;
  double wl = 0.0;
  for (int y = 0; y < n; ++y)
  {
    const double wr = (double)J.col_w[(size_t)(y + 1) * W + x];
    const float2 r = J.rowres[(size_t)y * W + x];
    const double a = -lam * wl;
    const double b = 1.0 + lam * (wl + wr);
    const double c = -lam * wr;
    const double inv = 1.0 / (b - fc * a);
    fc = c * inv;
    fd = ((double)r.x - fd * a) * inv;
    fi = ((double)r.y - fi * a) * inv;
    const size_t o = (size_t)y * W + x;
    tc[o] = fc;
    td[o] = fd;
    ti[o] = fi;
    wl = wr;
  }
  double nd = 0.0, ni = 0.0;
  for (int y = n - 1; y >= 0; --y)
  {
    const size_t o = (size_t)y * W + x;
    const double cc = tc[o];
    nd = td[o] - cc * nd;
    ni = ti[o] - cc * ni;
    J.dense[o] = (float)(nd / ni);
  }
}

} // namespace

void launch_weights(const Batch &B, int blocks, KParams kp,
                    int arith, cudaStream_t s)
{
  if (arith == QM_ARITH_IEEE)
    k_weights<ArithIeee><<<blocks, kFlatThreads, 0, s>>>(B, kp);
  else
    k_weights<ArithRef><<<blocks, kFlatThreads, 0, s>>>(B, kp);
}

void launch_row_solve(const Batch &B, int blocks, KParams kp,
                      cudaStream_t s)
{
  k_row_solve<<<blocks, kLineThreads, 0, s>>>(B, kp);
}

void launch_col_solve(const Batch &B, int blocks, KParams kp,
                      cudaStream_t s)
{
  k_col_solve<<<blocks, kLineThreads, 0, s>>>(B, kp);
}

} // namespace qm
