// Internal device-side definitions of the depth pipeline.
//
// A batch is a list of keyframe jobs (one per camera stream) of possibly
// different image sizes, hypothesis and slot counts.  Every stage runs as ONE
// kernel launch over all jobs: the host precomputes, per stage, the prefix sum
// of the blocks each job needs (`prefix[j] .. prefix[j+1]`), and a block finds
// its job by binary search over that prefix.
//
// This translation-unit family is compiled with -ftz=true -prec-div=false
// -prec-sqrt=false -fmad=true: the single-precision `/`, sqrtf and rsqrtf and
// the multiply-add contraction are then the ones the reference build gets
// from -use_fast_math.  The reference-arithmetic code paths below are written
// in the same expression forms as the reference's PinholeCamera / SE3 /
// helper_math code so that the compiler produces the same roundings (bit-exact
// costs and labels versus the reference kernels); the IEEE paths spell every
// operation with a round-to-nearest intrinsic (never contracted), which is
// what the CPU oracle computes.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "qm_capi.h"

namespace qm
{

constexpr int kMaxLevels = QM_MAX_BP_LEVELS;
constexpr int kMaxSlots = QM_MAX_SLOTS;
constexpr int kWarp = 32;

// Message directions, in the order of the messages' storage.
enum Dir
{
  kUp = 0,   // message a cell sends to its upper neighbour
  kDown = 1, // ... to its lower neighbour
  kLeft = 2, // ... to its left neighbour
  kRight = 3 // ... to its right neighbour
};

struct LevelDesc
{
  int w, h;       // cells at this pyramid level
  float *data;    // [h][w][D] data cost
  float *msg[4];  // [h][w][D] outgoing messages, by Dir
};

struct JobDesc
{
  // geometry and hypotheses
  int W, H, D, F;
  int cw, ch;
  float fx, fy, cx, cy;
  double min_inv, step;
  // inputs
  const uint8_t *ref;
  int ref_pitch;
  int slot_base; // first entry of this job in the slot tables
  int slot_pitch;
  // pipeline buffers
  uint8_t *levels; // W*H quadtree level per pixel
  int nlev;
  LevelDesc lv[kMaxLevels];
  int32_t *labels; // cw*ch or null
  float *sparse;   // W*H sparse depth (the reference's debug image)
  float *dense;    // W*H upsampled depth, fused in place
  float2 *rowres;  // W*H row-smoothed (depth, indicator)
  float4 *seeds_in;
  float4 *seeds_out;
  unsigned long long *zkey; // W*H z-buffer keys (all ones = empty; the row
                            // solve resets them when non-null)
  int32_t *table;           // W*H fusion source index (0 = none)
  float Tf[12];             // T_income<-lastfuse
  int keep_sparse;          // 1: `sparse` already holds this frame's
                            // semi-dense depths (the quadtree pass keeps them)
};

// The jobs of one launch.  Batched runs keep the job array, the per-stage
// block prefix and the slot tables in device memory; single-keyframe stage
// calls carry their one job (and its slots) inline in the kernel parameter,
// so those calls need no device allocation.
// Measurement slots of a job after merging duplicates: a slot that appears
// k times (same image, same pose) is evaluated once with weight k.  The SAD
// and the valid count are integers, so the weighted sums equal the
// reference's per-slot sums exactly.
struct SlotInline
{
  const uint8_t *ptr[kMaxSlots];
  float T[kMaxSlots * 12];
  int w[kMaxSlots];
};

struct Batch
{
  const JobDesc *jobs; // null: the single job `one`
  const int *prefix;   // block prefix of this stage over the jobs
  int njobs;
  int block0;  // global block index of this launch's first block (job groups)
  int uniform; // > 0: every job has this many blocks (job = block / uniform)
  int rev;     // 1: blocks take their work in reverse order (last block first)
  const uint8_t *const *slot_ptr; // per slot, device image (null: `slots`)
  const float *slot_T;            // per slot, 12 floats T_slot<-ref
  const int *slot_w;              // per slot, multiplicity
  JobDesc one;
  SlotInline slots;
};

// Parameters shared by all jobs of a batch (kernel arguments by value).
struct KParams
{
  float P1, P2;
  int qt_max, qt_min;
  float qt_thr;
  double up_sigma, up_lambda;
};

__device__ __forceinline__ int find_job(const int *__restrict__ prefix, int njobs, int block)
{
  int lo = 0, hi = njobs - 1;
  while (lo < hi)
  {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(prefix + mid) <= block)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// The job of this block and the block's index inside that job.  A launch may
// cover a contiguous group of jobs only: its blocks then start at block0.
__device__ __forceinline__ const JobDesc &job_of(const Batch &B, int &local_block)
{
  const int block =
      (B.rev ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x) + B.block0;
  if (B.jobs == nullptr)
  {
    local_block = block;
    return B.one;
  }
  if (B.uniform > 0)
  {
    const int j = block / B.uniform;
    local_block = block - j * B.uniform;
    return B.jobs[j];
  }
  const int j = find_job(B.prefix, B.njobs, block);
  local_block = block - __ldg(B.prefix + j);
  return B.jobs[j];
}

__device__ __forceinline__ const uint8_t *slot_image(const Batch &B, int slot)
{
  return B.slot_ptr ? B.slot_ptr[slot] : B.slots.ptr[slot];
}

__device__ __forceinline__ const float *slot_pose(const Batch &B, int slot)
{
  return B.slot_ptr ? B.slot_T + 12 * slot : B.slots.T + 12 * slot;
}

__device__ __forceinline__ int slot_weight(const Batch &B, int slot)
{
  return B.slot_ptr ? B.slot_w[slot] : B.slots.w[slot];
}

// Double -> int by truncation toward zero with saturation (C conversion as
// the reference performs it on `float + 0.5`).
__device__ __forceinline__ int trunc_int(double v) { return (int)v; }

struct Cam
{
  float fx, fy, cx, cy;
};

// ---------------------------------------------------------------------------
// Arithmetic policies.  Ref = the reference's fast-math forms; Ieee = correctly
// rounded operations in the order the oracle uses.

struct ArithRef
{
  static constexpr bool kIeee = false;
  // normalize(cam2world(x, y)): helper_math.h normalize, pinhole_camera.cuh:48-52
  static __device__ __forceinline__ float3 ray(float x, float y, const Cam &c)
  {
    float3 v = make_float3((x - c.cx) / c.fx, (y - c.cy) / c.fy, 1.0f);
    float inv = rsqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    return make_float3(v.x * inv, v.y * inv, v.z * inv);
  }
  static __device__ __forceinline__ float3 scale(float3 d, float s)
  {
    return make_float3(d.x * s, d.y * s, d.z * s);
  }
  // SE3<float> * p: rotate then translate (se3.cuh:121-151,197-201)
  static __device__ __forceinline__ float3 apply(const float *T, float3 p)
  {
    float3 r = make_float3(T[0] * p.x + T[1] * p.y + T[2] * p.z,
                           T[4] * p.x + T[5] * p.y + T[6] * p.z,
                           T[8] * p.x + T[9] * p.y + T[10] * p.z);
    return make_float3(r.x + T[3], r.y + T[7], r.z + T[11]);
  }
  // PinholeCamera::world2cam (pinhole_camera.cuh:57-61)
  static __device__ __forceinline__ float2 project(float3 q, const Cam &c)
  {
    return make_float2(c.fx * q.x / q.z + c.cx, c.fy * q.y / q.z + c.cy);
  }
  static __device__ __forceinline__ float hyp_depth(double step, double mn, int d)
  {
    return 1.0 / (step * d + mn);
  }
  // my_depth_cost / (float)aggregate_num / 255.0f (depth_extract.cu:223)
  static __device__ __forceinline__ float sad_norm(float sad, float n) { return sad / n / 255.0f; }
  static __device__ __forceinline__ float length(float3 p) { return sqrtf(p.x * p.x + p.y * p.y + p.z * p.z); }
  static __device__ __forceinline__ float div(float a, float b) { return a / b; }
  static __device__ __forceinline__ float exp(float a) { return __expf(a); }
};

struct ArithIeee
{
  static constexpr bool kIeee = true;
  static __device__ __forceinline__ float3 ray(float x, float y, const Cam &c)
  {
    const float vx = __fdiv_rn(__fsub_rn(x, c.cx), c.fx);
    const float vy = __fdiv_rn(__fsub_rn(y, c.cy), c.fy);
    const float vz = 1.0f;
    const float dot = __fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)), __fmul_rn(vz, vz));
    const float inv = __fdiv_rn(1.0f, __fsqrt_rn(dot));
    return make_float3(__fmul_rn(vx, inv), __fmul_rn(vy, inv), __fmul_rn(vz, inv));
  }
  static __device__ __forceinline__ float3 scale(float3 d, float s)
  {
    return make_float3(__fmul_rn(d.x, s), __fmul_rn(d.y, s), __fmul_rn(d.z, s));
  }
  static __device__ __forceinline__ float row(const float *T, int r, float3 p)
  {
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(T[4 * r], p.x), __fmul_rn(T[4 * r + 1], p.y)),
                               __fmul_rn(T[4 * r + 2], p.z)),
                     T[4 * r + 3]);
  }
  static __device__ __forceinline__ float3 apply(const float *T, float3 p)
  {
    return make_float3(row(T, 0, p), row(T, 1, p), row(T, 2, p));
  }
  static __device__ __forceinline__ float2 project(float3 q, const Cam &c)
  {
    return make_float2(__fadd_rn(__fdiv_rn(__fmul_rn(c.fx, q.x), q.z), c.cx),
                       __fadd_rn(__fdiv_rn(__fmul_rn(c.fy, q.y), q.z), c.cy));
  }
  static __device__ __forceinline__ float hyp_depth(double step, double mn, int d)
  {
    return (float)__ddiv_rn(1.0, __dadd_rn(__dmul_rn(step, (double)d), mn));
  }
  static __device__ __forceinline__ float sad_norm(float sad, float n)
  {
    return __fdiv_rn(__fdiv_rn(sad, n), 255.0f);
  }
  static __device__ __forceinline__ float length(float3 p)
  {
    return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(p.x, p.x), __fmul_rn(p.y, p.y)), __fmul_rn(p.z, p.z)));
  }
  static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
  static __device__ __forceinline__ float exp(float a) { return expf(a); }
};

// ---------------------------------------------------------------------------
// Warp helpers

__device__ __forceinline__ float warp_min(float v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

} // namespace qm
