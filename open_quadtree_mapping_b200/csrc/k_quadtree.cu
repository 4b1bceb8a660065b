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
    if (J.sparse && !J.keep_sparse)
      J.sparse[(size_t)y * J.W + x] = 0.0f; // the debug image starts empty

  }
}

// Summary of an aligned block: intensity sum, max, min, and whether it is
// complete (inside the image) with every sub-block approved.
struct Node
{
  int sum, mx, mn;
  bool ok;
};

__device__ __forceinline__ Node merge(Node a, Node b)
{
  return Node{a.sum + b.sum, max(a.mx, b.mx), min(a.mn, b.mn), a.ok && b.ok};
}

__device__ __forceinline__ Node merge_lane(Node a, int lane_xor)
{
  Node b;
  b.sum = __shfl_xor_sync(0xffffffffu, a.sum, lane_xor);
  b.mx = __shfl_xor_sync(0xffffffffu, a.mx, lane_xor);
  b.mn = __shfl_xor_sync(0xffffffffu, a.mn, lane_xor);
  b.ok = __shfl_xor_sync(0xffffffffu, a.ok ? 1 : 0, lane_xor) != 0;
  return merge(a, b);
}

// approval of a complete block of 4^i pixels (same arithmetic as above)
__device__ __forceinline__ bool approve(const Node &n, int i, float thr)
{
  if (!n.ok)
    return false;
  const float mean = (float)n.sum * (1.0f / (float)(1 << (2 * i)));
  return ((float)n.mx - mean <= thr) && (mean - (float)n.mn <= thr);
}

constexpr int kQtWarps = 8;

// The default 16 x 16 tile (qt_max = 4), one warp per tile and no shared
// memory: lane (a, b) = (lane & 3, lane >> 2) owns the 4 x 2 pixels at
// columns 4a..4a+3, rows 2b, 2b+1 -- two 2x2 blocks of level 1.  Level 2
// joins lanes b ^ 1 (lane ^ 4), level 3 lanes a ^ 1 and b ^ 2 (lane ^ 1,
// ^ 8), level 4 lanes a ^ 2 and b ^ 4 (lane ^ 2, ^ 16).  Results equal the
// general kernel's (integer sums and extrema, the same float test).
__global__ void __launch_bounds__(kQtWarps * 32)
    k_quadtree16(const __grid_constant__ Batch B, KParams kp)
{
  int lb;
  const JobDesc &J = job_of(B, lb);
  const int W = J.W, H = J.H;
  const int tiles_x = (W + 15) >> 4;
  const int tile = lb * kQtWarps + (threadIdx.x >> 5);
  if (tile >= tiles_x * ((H + 15) >> 4))
    return;
  const int lane = threadIdx.x & 31, a = lane & 3, b = lane >> 2;
  const int x0 = (tile % tiles_x) * 16 + 4 * a, y0 = (tile / tiles_x) * 16 + 2 * b;
  int v[2][4];
  bool in[2][4];
  // the lane's 4 bytes of a row as one 32-bit load when the row segment is
  // inside the image and 4-byte aligned (every batched frame: W % 16 == 0)
  const bool wide = x0 + 3 < W && (J.ref_pitch & 3) == 0 && ((uintptr_t)J.ref & 3) == 0;
#pragma unroll
  for (int r = 0; r < 2; ++r)
  {
    const uint8_t *row = J.ref + (size_t)(y0 + r) * J.ref_pitch + x0;
    if (wide && y0 + r < H)
    {
      const unsigned q = *reinterpret_cast<const unsigned *>(row);
#pragma unroll
      for (int c = 0; c < 4; ++c)
      {
        in[r][c] = true;
        v[r][c] = (int)((q >> (8 * c)) & 0xffu);
      }
    }
    else
#pragma unroll
      for (int c = 0; c < 4; ++c)
      {
        in[r][c] = x0 + c < W && y0 + r < H;
        v[r][c] = in[r][c] ? (int)row[c] : 0;
      }
  }
  // level 1: the lane's two 2x2 blocks
  Node n1[2];
  bool ok1[2];
#pragma unroll
  for (int k = 0; k < 2; ++k)
  {
    Node n{0, 0, 255, true};
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int c = 2 * k; c < 2 * k + 2; ++c)
      {
        n.sum += v[r][c];
        n.mx = max(n.mx, v[r][c]);
        n.mn = min(n.mn, v[r][c]);
        n.ok = n.ok && in[r][c];
      }
    ok1[k] = approve(n, 1, kp.qt_thr);
    n1[k] = Node{n.sum, n.mx, n.mn, ok1[k]};
  }
  Node n2 = merge(n1[0], n1[1]);
  n2 = merge_lane(n2, 4);
  const bool ok2 = approve(n2, 2, kp.qt_thr);
  n2.ok = ok2;
  Node n3 = merge_lane(merge_lane(n2, 1), 8);
  const bool ok3 = approve(n3, 3, kp.qt_thr);
  n3.ok = ok3;
  Node n4 = merge_lane(merge_lane(n3, 2), 16);
  const bool ok4 = approve(n4, 4, kp.qt_thr);
  const int upper = ok4 ? 4 : ok3 ? 3 : ok2 ? 2 : 1;
  const bool clear = J.sparse && !J.keep_sparse; // the debug image starts empty
#pragma unroll
  for (int r = 0; r < 2; ++r)
  {
    if (y0 + r >= H)
      continue;
    const size_t o = (size_t)(y0 + r) * W + x0;
    // four levels as one 32-bit store and four depths as one 16-byte store
    // when the row segment is inside the image and aligned (the level map
    // and the sparse image are W-pitched)
    const bool seg = x0 + 3 < W && (W & 3) == 0;
    if (seg && ((uintptr_t)J.levels & 3) == 0 &&
        (!clear || ((uintptr_t)J.sparse & 15) == 0))
    {
      unsigned q = 0;
#pragma unroll
      for (int c = 0; c < 4; ++c)
        q |= (unsigned)max(ok1[c >> 1] ? upper : 0, kp.qt_min) << (8 * c);
      *reinterpret_cast<unsigned *>(J.levels + o) = q;
      if (clear)
        *reinterpret_cast<float4 *>(J.sparse + o) = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      continue;
    }
#pragma unroll
    for (int c = 0; c < 4; ++c)
    {
      if (!in[r][c])
        continue;
      const int level = ok1[c >> 1] ? upper : 0;
      J.levels[o + c] = (uint8_t)max(level, kp.qt_min);
      if (clear)
        J.sparse[o + c] = 0.0f;
    }
  }
}

} // namespace

int quadtree_blocks(int W, int H, int qt_max)
{
  const int T = 1 << qt_max;
  const int tiles = ((W + T - 1) / T) * ((H + T - 1) / T);
  return qt_max == 4 ? (tiles + kQtWarps - 1) / kQtWarps : tiles;
}

void launch_quadtree(const Batch &B, int blocks, KParams kp, cudaStream_t s)
{
  if (kp.qt_max == 4)
    k_quadtree16<<<blocks, kQtWarps * 32, 0, s>>>(B, kp);
  else
    k_quadtree<<<blocks, 256, 0, s>>>(B, kp);
}

} // namespace qm
