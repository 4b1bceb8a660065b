// Quadtree levels from intensity uniformity (quadtree_image_kernal,
// quadtree.cu:17-77 of the reference).
//
// One CTA per tile of 2^qt_max x 2^qt_max pixels.  Level by level, each
// aligned block of side 2^i gets (sum, max, min, approved) from its four
// children in shared memory; a block is approved when it is complete (inside
// the image), its children are approved and max - mean <= thr and
// mean - min <= thr (equivalently |I - mean| <= thr for every pixel, the
// reference's test).  Intensities are integers, sums of up to 4^qt_max of them
// are exact and the mean divides by a power of two, so every comparison is
// exact and independent of summation order.  A pixel's level is the largest
// approved level, clamped to at least qt_min.
//
// Bytes per pixel: 1 read (u8 image) + 1 written (u8 level).
#include "launch.h"

namespace qm
{

namespace
{

constexpr int kMaxTile = 32;

__global__ void __launch_bounds__(256)
    k_quadtree(const __grid_constant__ Batch B, KParams kp)
{
  int tile;
  const JobDesc &J = job_of(B, tile);
  const int T = 1 << kp.qt_max;
  const int tiles_x = (J.W + T - 1) / T;
  const int x0 = (tile % tiles_x) * T, y0 = (tile / tiles_x) * T;
  const int nthreads = blockDim.x;

  __shared__ int s_sum[2][kMaxTile * kMaxTile];
  __shared__ short s_max[2][kMaxTile * kMaxTile];
  __shared__ short s_min[2][kMaxTile * kMaxTile];
  __shared__ unsigned char s_ok[2][kMaxTile * kMaxTile];
  // approved flag of every block of every level, level i at offset off[i]
  __shared__ unsigned char s_appr[kMaxTile * kMaxTile * 2];

  // level 0: pixels
  for (int p = threadIdx.x; p < T * T; p += nthreads)
  {
    const int x = x0 + (p % T), y = y0 + (p / T);
    const bool in = x < J.W && y < J.H;
    const int v = in ? (int)J.ref[(size_t)y * J.ref_pitch + x] : 0;
    s_sum[0][p] = v;
    s_max[0][p] = (short)v;
    s_min[0][p] = (short)v;
    s_ok[0][p] = in ? 1 : 0;
  }
  __syncthreads();
  int cur = 0;
  int off = 0;
  for (int i = 1; i <= kp.qt_max; ++i)
  {
    const int side = T >> i; // blocks per row at level i
    const int nb = side * side;
    const int cside = side * 2;
    for (int b = threadIdx.x; b < nb; b += nthreads)
    {
      const int bx = b % side, by = b / side;
      int sum = 0, mx = 0, mn = 255;
      bool ok = true;
#pragma unroll
      for (int c = 0; c < 4; ++c)
      {
        const int ci = (2 * by + (c >> 1)) * cside + (2 * bx + (c & 1));
        sum += s_sum[cur][ci];
        mx = max(mx, (int)s_max[cur][ci]);
        mn = min(mn, (int)s_min[cur][ci]);
        ok = ok && s_ok[cur][ci];
      }
      if (ok)
      {
        const float mean = (float)sum * (1.0f / (float)(1 << (2 * i)));
        ok = ((float)mx - mean <= kp.qt_thr) && (mean - (float)mn <= kp.qt_thr);
      }
      s_sum[cur ^ 1][b] = sum;
      s_max[cur ^ 1][b] = (short)mx;
      s_min[cur ^ 1][b] = (short)mn;
      s_ok[cur ^ 1][b] = ok ? 1 : 0;
      s_appr[off + b] = ok ? 1 : 0;
    }
    off += nb;
    cur ^= 1;
    __syncthreads();
  }
  for (int p = threadIdx.x; p < T * T; p += nthreads)
  {
    const int px = p % T, py = p / T;
    const int x = x0 + px, y = y0 + py;
    if (x >= J.W || y >= J.H)
      continue;
    int level = 0, o = 0;
    for (int i = 1; i <= kp.qt_max; ++i)
    {
      const int side = T >> i;
      if (!s_appr[o + (py >> i) * side + (px >> i)])
        break;
      level = i;
      o += side * side;
    }
    J.levels[(size_t)y * J.W + x] = (uint8_t)max(level, kp.qt_min);
    if (J.sparse)
      J.sparse[(size_t)y * J.W + x] = 0.0f; // the debug image starts empty

  }
}

} // namespace

int quadtree_tile(int qt_max) { return 1 << qt_max; }

void launch_quadtree(const Batch &B, int blocks, KParams kp, cudaStream_t s)
{
  k_quadtree<<<blocks, 256, 0, s>>>(B, kp);
}

} // namespace qm
