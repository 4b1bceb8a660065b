// Point cloud of a fused depth map: the loop of Publisher::publishPointCloud
// (publisher.cpp:129-166) on the device.  Every pixel whose depth is not
// below 0.1 becomes the point T_world_ref * (normalize(((x - cx) / fx,
// (y - cy) / fy, 1)) * depth) with the reference image's intensity, and the
// points keep the row-major pixel order of the reference's push_back loop.
//
// The reference runs this loop on the host (g++, no FMA contraction on
// x86-64, helper_math.h's host rsqrtf = 1 / sqrtf), so every operation here
// is an explicitly IEEE-rounded single operation in the same order: the
// points are bit-identical to the host loop's.
//
// Three launches, no waits between blocks: per-tile counts, one scan block
// over the tile counts (also writing the total), and the order-preserving
// write.  A tile is 1024 consecutive pixels; thread t of a block holds pixels
// t, t + 256, t + 512 and t + 768 of its tile, so depth and image loads are
// coalesced along the rows.  Bytes per pixel: 4 (depth) read twice, 1 (image)
// read once, 16 written per point.
#include "launch.h"

namespace qm
{

namespace
{

constexpr int kPcThreads = 256;
constexpr int kPcPer = 4;
constexpr int kPcTile = kPcThreads * kPcPer;
constexpr int kScanThreads = 1024;

struct PcArgs
{
  const float *depth;
  size_t stride; // floats
  const uint8_t *ref;
  size_t pitch; // bytes
  int W, H;
  float fx, fy, cx, cy;
  float T[12];
  float4 *out;
  int *tile_off; // per tile: count, then exclusive offset
  int *total;
  int tiles;
};

// publisher.cpp:150: `depth_value < 0.1` compares the float promoted to
// double; for floats that is the same test as d < 0.1f.
__device__ __forceinline__ bool pc_keep(float d) { return !(d < 0.1f); }

__device__ __forceinline__ float pc_depth(const PcArgs &a, long p, int &x, int &y)
{
  y = (int)(p / a.W);
  x = (int)(p - (long)y * a.W);
  return a.depth[(size_t)y * a.stride + x];
}

__device__ __forceinline__ float4 pc_point(const PcArgs &a, int x, int y, float d)
{
  // make_float3((x - cx) / fx, (y - cy) / fy, 1.0f), publisher.cpp:152
  const float u = __fdiv_rn(__fsub_rn((float)x, a.cx), a.fx);
  const float v = __fdiv_rn(__fsub_rn((float)y, a.cy), a.fy);
  // normalize: v * (1 / sqrt(dot(v, v))), helper_math.h:62-65,1278-1281,1364-1368
  const float n2 = __fadd_rn(__fadd_rn(__fmul_rn(u, u), __fmul_rn(v, v)), 1.0f);
  const float inv = __fdiv_rn(1.0f, __fsqrt_rn(n2));
  // f * depth_value, then SE3 rotate + translate (se3.cuh:122-127,146-151,198-201)
  const float px = __fmul_rn(__fmul_rn(u, inv), d);
  const float py = __fmul_rn(__fmul_rn(v, inv), d);
  const float pz = __fmul_rn(inv, d);
  const float *T = a.T;
  auto row = [&](int r) {
    const float s = __fadd_rn(__fadd_rn(__fmul_rn(T[4 * r], px), __fmul_rn(T[4 * r + 1], py)),
                              __fmul_rn(T[4 * r + 2], pz));
    return __fadd_rn(s, T[4 * r + 3]);
  };
  return make_float4(row(0), row(1), row(2), (float)a.ref[(size_t)y * a.pitch + x]);
}

__global__ void __launch_bounds__(kPcThreads) k_pc_count(const __grid_constant__ PcArgs a)
{
  __shared__ int warp_sum[kPcThreads / 32];
  const long n = (long)a.W * a.H;
  const long base = (long)blockIdx.x * kPcTile;
  int c = 0;
#pragma unroll
  for (int k = 0; k < kPcPer; ++k)
  {
    const long p = base + k * kPcThreads + threadIdx.x;
    int x, y;
    if (p < n && pc_keep(pc_depth(a, p, x, y)))
      ++c;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0)
    warp_sum[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0)
  {
    int s = 0;
    for (int w = 0; w < kPcThreads / 32; ++w)
      s += warp_sum[w];
    a.tile_off[blockIdx.x] = s;
  }
}

// One block: exclusive scan of the tile counts in place, total to *a.total.
__global__ void __launch_bounds__(kScanThreads) k_pc_scan(const __grid_constant__ PcArgs a)
{
  __shared__ int part[kScanThreads];
  const int per = (a.tiles + kScanThreads - 1) / kScanThreads;
  const int b0 = threadIdx.x * per;
  const int b1 = min(a.tiles, b0 + per);
  int s = 0;
  for (int b = b0; b < b1; ++b)
    s += a.tile_off[b];
  part[threadIdx.x] = s;
  __syncthreads();
  // Hillis-Steele inclusive scan of the per-thread sums
  for (int o = 1; o < kScanThreads; o <<= 1)
  {
    const int v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int run = part[threadIdx.x] - s;
  for (int b = b0; b < b1; ++b)
  {
    const int c = a.tile_off[b];
    a.tile_off[b] = run;
    run += c;
  }
  if (threadIdx.x == kScanThreads - 1)
    *a.total = part[kScanThreads - 1];
}

__global__ void __launch_bounds__(kPcThreads) k_pc_write(const __grid_constant__ PcArgs a)
{
  __shared__ int warp_sum[kPcThreads / 32];
  const long n = (long)a.W * a.H;
  const long base = (long)blockIdx.x * kPcTile;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int run = a.tile_off[blockIdx.x];
  for (int k = 0; k < kPcPer; ++k)
  {
    const long p = base + k * kPcThreads + threadIdx.x;
    int x = 0, y = 0;
    float d = 0.0f;
    bool keep = false;
    if (p < n)
    {
      d = pc_depth(a, p, x, y);
      keep = pc_keep(d);
    }
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if (lane == 0)
      warp_sum[warp] = __popc(m);
    __syncthreads();
    int before = 0, all = 0;
    for (int w = 0; w < kPcThreads / 32; ++w)
    {
      const int c = warp_sum[w];
      before += w < warp ? c : 0;
      all += c;
    }
    if (keep)
      a.out[run + before + __popc(m & ((1u << lane) - 1u))] = pc_point(a, x, y, d);
    run += all;
    __syncthreads(); // warp_sum is rewritten by the next k
  }
}

PcArgs pc_args(const float *depth, size_t stride, const uint8_t *ref, size_t pitch, int W, int H,
               const Cam &cam, const float *T, float4 *out, void *ws)
{
  PcArgs a;
  a.depth = depth;
  a.stride = stride;
  a.ref = ref;
  a.pitch = pitch;
  a.W = W;
  a.H = H;
  a.fx = cam.fx;
  a.fy = cam.fy;
  a.cx = cam.cx;
  a.cy = cam.cy;
  for (int k = 0; k < 12; ++k)
    a.T[k] = T[k];
  a.out = out;
  a.tiles = point_cloud_tiles(W, H);
  a.total = (int *)ws;
  a.tile_off = (int *)ws + 1;
  return a;
}

} // namespace

int point_cloud_tiles(int W, int H) { return (int)(((long)W * H + kPcTile - 1) / kPcTile); }

size_t point_cloud_workspace(int W, int H) { return sizeof(int) * (1 + (size_t)point_cloud_tiles(W, H)); }

void launch_point_cloud(const float *depth, size_t stride, const uint8_t *ref, size_t pitch, int W,
                        int H, const Cam &cam, const float *T_world_ref, float4 *out, int *count,
                        void *ws, cudaStream_t s)
{
  PcArgs a = pc_args(depth, stride, ref, pitch, W, H, cam, T_world_ref, out, ws);
  a.total = count ? count : a.total;
  k_pc_count<<<a.tiles, kPcThreads, 0, s>>>(a);
  k_pc_scan<<<1, kScanThreads, 0, s>>>(a);
  k_pc_write<<<a.tiles, kPcThreads, 0, s>>>(a);
}

} // namespace qm
