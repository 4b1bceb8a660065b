// Test infrastructure only: the reference comparator.
//
// This translation unit compiles the reference's own depth-path kernels,
// unmodified, from the reference source tree (src/quadtree.cu,
// src/depth_extract.cu, src/bpextract.cu, src/depth_upsample.cu,
// src/depth_fusion.cu, and for the semi-dense tracker src/seed_init.cu and
// src/lsd_semidense.cu, are #included by path; see oracle/Makefile), with the
// reference's flags (-O3 -use_fast_math) for sm_100a.  Only the legacy texture
// references are swapped for texture objects (ref_shim/quadmap/
// texture_memory.cuh) and <opencv2/opencv.hpp> for an empty header.  The
// same file also builds the patched variants (other DEPTH_NUM and inverse-
// depth range, oracle/refpatch.py): every per-hypothesis launch below takes
// DEPTH_NUM threads where the reference's host code writes 64, which is the
// reference's own launch when DEPTH_NUM is 64.
//
// The extern "C" functions below replay the host sequences of
// SeedMatrix::extract_depth (src/seed_matrix.cu:448-551) and
// SeedMatrix::fuse_output_depth (src/seed_matrix.cu:553-597) on host buffers,
// so tests can dump every intermediate (level map, cost volume, final BP
// messages, sparse depth, upsampled depth, fused depth and seeds) and the
// bench can time the reference kernels on the same inputs.  Nothing in the
// product links this library.
#include <cuda_runtime.h>
#include <chrono>
#include <cstring>
#include <vector>

#include <quadmap/pixel_cost.cuh>
#include <quadmap/device_image.cuh>
#include <quadmap/se3.cuh>
#include <quadmap/camera_model/pinhole_camera.cuh>
#include <quadmap/match_parameter.cuh>
#include <quadmap/texture_memory.cuh>
#include <quadmap/stereo_parameter.cuh>
#include <quadmap/DepthSeed.cuh>

#include "seed_init.cu"
#include "lsd_semidense.cu"
#include "quadtree.cu"
#include "depth_extract.cu"
#include "bpextract.cu"
#include "depth_upsample.cu"
#include "depth_fusion.cu"

using namespace quadmap;

namespace
{

int g_err = 0;

SE3<float> se3_from(const float *t12)
{
  SE3<float> s;
  for (int i = 0; i < 12; ++i)
    s.data[i] = t12[i];
  return s;
}

template <typename T>
void download(const DeviceImage<T> &img, T *out)
{
  if (out)
    img.getDevData(out);
}

// The hierarchical BP of bpextract.cu:37-167, replayed kernel for kernel with
// the same launch shapes, except that the level-0 messages are kept so that
// the winning labels can be recomputed from them by the caller.
void bp_keep_messages(DeviceImage<PIXEL_COST> &image_cost_map, float *msg_out)
{
  const int width = image_cost_map.width;
  const int height = image_cost_map.height;
  const int hbp_level = 4;
  int hbp_iterate[4] = {4, 10, 10, 10};
  int h_width[4], h_height[4];
  h_width[0] = width;
  h_height[0] = height;
  for (int i = 1; i < hbp_level; i++)
  {
    h_width[i] = (h_width[i - 1] + 1) / 2;
    h_height[i] = (h_height[i - 1] + 1) / 2;
  }
  DeviceImage<PIXEL_COST> *pyr[4];
  pyr[0] = &image_cost_map;
  for (int i = 1; i < hbp_level; i++)
    pyr[i] = new DeviceImage<PIXEL_COST>(h_width[i], h_height[i]);
  // bpextract.cu:67-78; with more than 64 hypotheses (a patched build)
  // the z extent is split over DEPTH_NUM / 64 blocks
  dim3 hb;
  hb.z = 64;
  for (int i = 1; i < hbp_level; i++)
  {
    dim3 hg(h_width[i], h_height[i], DEPTH_NUM / 64);
    cost_distribute<<<hg, hb>>>(pyr[i - 1]->dev_ptr, pyr[i]->dev_ptr);
    cudaDeviceSynchronize();
  }
  DeviceImage<PIXEL_COST> *msg[4];
  for (int m = 0; m < 4; ++m)
  {
    msg[m] = new DeviceImage<PIXEL_COST>(h_width[hbp_level - 1], h_height[hbp_level - 1]);
    msg[m]->zero();
  }
  for (int lv = hbp_level - 1; lv >= 0; lv--)
  {
    if (lv < hbp_level - 1)
    {
      DeviceImage<PIXEL_COST> *next[4];
      for (int m = 0; m < 4; ++m)
        next[m] = new DeviceImage<PIXEL_COST>(h_width[lv], h_height[lv]);
      dim3 ub(DEPTH_NUM);
      dim3 ug(h_width[lv + 1], h_height[lv + 1]);
      for (int m = 0; m < 4; m++)
        upsample<<<ug, ub>>>(msg[m]->dev_ptr, next[m]->dev_ptr);
      cudaDeviceSynchronize();
      for (int m = 0; m < 4; m++)
      {
        delete msg[m];
        msg[m] = next[m];
      }
    }
    dim3 bb(4, DEPTH_NUM);
    dim3 bg((h_width[lv] + 1) / 2, h_height[lv]);
    bool A_set = true;
    for (int it = 0; it < hbp_iterate[lv]; it++)
    {
      bp<<<bg, bb>>>(pyr[lv]->dev_ptr, msg[0]->dev_ptr, msg[1]->dev_ptr, msg[2]->dev_ptr,
                     msg[3]->dev_ptr, A_set, lv + 2);
      A_set = !A_set;
      cudaDeviceSynchronize();
    }
  }
  // bp() argument order is (data, lm, rm, up, dm): msg[0]=left, msg[1]=right,
  // msg[2]=up, msg[3]=down.  Dump as up, down, left, right.
  if (msg_out)
  {
    const size_t n = (size_t)width * height * DEPTH_NUM;
    msg[2]->getDevData(reinterpret_cast<PIXEL_COST *>(msg_out + 0 * n));
    msg[3]->getDevData(reinterpret_cast<PIXEL_COST *>(msg_out + 1 * n));
    msg[0]->getDevData(reinterpret_cast<PIXEL_COST *>(msg_out + 2 * n));
    msg[1]->getDevData(reinterpret_cast<PIXEL_COST *>(msg_out + 3 * n));
  }
  for (int i = 1; i < hbp_level; i++)
    delete pyr[i];
  for (int m = 0; m < 4; ++m)
    delete msg[m];
}

struct ExtractState
{
  int w, h;
  PinholeCamera cam;
  DeviceImage<float> income;
  DeviceImage<int> age;
  std::vector<DeviceImage<float> *> frames;
  MatchParameter mp;
  ExtractState(int w_, int h_, const PinholeCamera &c)
      : w(w_), h(h_), cam(c), income(w_, h_), age(w_, h_)
  {
    age.zero();
  }
  ~ExtractState()
  {
    for (auto *f : frames)
      delete f;
    if (mp.is_dev_allocated)
      cudaFree(mp.dev_ptr);
  }
};

// SeedMatrix::extract_depth (seed_matrix.cu:448-551) on the given state;
// debug_image holds the sparse prior on entry and the BP depths on exit.
void run_extract(ExtractState &st, int nslots, DeviceImage<float> &debug_image,
                 DeviceImage<float> &depth_output, int *levels_out, float *cost_out,
                 float *msg_out)
{
  bindTexture(income_image_tex, st.income);
  st.mp.camera_model = st.cam;
  st.mp.current_frames = (int)st.frames.size();
  st.mp.setDevData();

  DeviceImage<int> quadtree_index(st.w, st.h);
  quadtree_index.zero();
  dim3 qb(16, 16);
  dim3 qg((st.w + 15) / 16, (st.h + 15) / 16);
  quadtree_image_kernal<<<qg, qb>>>(quadtree_index.dev_ptr);
  cudaDeviceSynchronize();
  bindTexture(quadtree_tex, quadtree_index, cudaFilterModePoint);

  DeviceImage<PIXEL_COST> image_cost(st.w / 4, st.h / 4);
  DeviceImage<int> add_num(st.w / 4, st.h / 4);
  image_cost.zero();
  add_num.zero();
  dim3 cb(DEPTH_NUM, nslots);
  dim3 cg(st.w / 4, st.h / 4);
  image_to_cost<<<cg, cb>>>(st.mp.dev_ptr, st.age.dev_ptr, image_cost.dev_ptr, add_num.dev_ptr);
  dim3 nb(DEPTH_NUM);
  normalize_the_cost<<<cg, nb>>>(image_cost.dev_ptr, add_num.dev_ptr);
  cudaDeviceSynchronize();

  download(quadtree_index, levels_out);
  if (cost_out)
    image_cost.getDevData(reinterpret_cast<PIXEL_COST *>(cost_out));
  if (msg_out)
  {
    // Same kernels on a copy of the cost volume, keeping the messages.
    DeviceImage<PIXEL_COST> cost_copy(st.w / 4, st.h / 4);
    cost_copy = image_cost;
    bp_keep_messages(cost_copy, msg_out);
  }
  bp_extract(image_cost, debug_image);
  global_upsample(debug_image, depth_output);
  cudaDeviceSynchronize();

  cudaUnbindTexture(quadtree_tex);
  cudaUnbindTexture(income_image_tex);
}

// SeedMatrix::fuse_output_depth (seed_matrix.cu:553-597).
void run_fuse(int w, int h, const PinholeCamera &cam, DeviceImage<float> &depth_output,
              DeviceImage<float4> &seeds, const SE3<float> &last_to_income,
              DeviceImage<int> *table_keep)
{
  DeviceImage<int> transform_table(w, h);
  DeviceImage<float4> new_seed(w, h);
  transform_table.zero();
  dim3 b(16, 16);
  dim3 g((w + 15) / 16, (h + 15) / 16);
  fuse_transform<<<g, b>>>(seeds.dev_ptr, transform_table.dev_ptr, last_to_income, cam);
  hole_filling<<<g, b>>>(transform_table.dev_ptr);
  fuse_currentmap<<<g, b>>>(transform_table.dev_ptr, depth_output.dev_ptr, seeds.dev_ptr,
                            new_seed.dev_ptr);
  seeds = new_seed;
  cudaDeviceSynchronize();
  if (table_keep)
    *table_keep = transform_table;
}

int status()
{
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess)
    return 100 + (int)e;
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return 100 + (int)e;
  return g_err;
}

} // namespace

extern "C" {

// The constants this build was compiled with: the reference's own
// (64, 0.01, (2.0 - 0.01) / 63) or a patched variant's (oracle/refpatch.py).
int qmref_depth_num() { return DEPTH_NUM; }
double qmref_min_inv_depth() { return MIN_INV_DEPTH; }
double qmref_inv_depth_step() { return STEP_INV_DEPTH; }

// Depth extraction as SeedMatrix::extract_depth does it.
//   income_img  w*h float (values 0..255)
//   frames_img  nframes*w*h float, ring order (index 0 = most recent)
//   T_frame_income  nframes*12 floats, row-major 3x4 T_frame<-income
//   nslots      measurement slots (blockDim.y of image_to_cost; reference 5;
//               DEPTH_NUM * nslots threads must fit one block, <= 1024)
//   debug_inout w*h: sparse prior in, sparse BP depth out
// Optional outputs (NULL to skip): levels (w*h int), cost ((w/4)*(h/4)*DEPTH_NUM),
// msg (4 x (w/4)*(h/4)*DEPTH_NUM, order up, down, left, right), dense (w*h).
int qmref_extract(int w, int h, float fx, float fy, float cx, float cy, const float *income_img,
                  int nframes, const float *frames_img, const float *T_frame_income, int nslots,
                  float *debug_inout, int *levels_out, float *cost_out, float *msg_out,
                  float *dense_out)
{
  if (nframes < 1 || nframes > KEYFRAME_NUM || nslots < 1 || nslots > 10 ||
      DEPTH_NUM * nslots > 1024)
    return 1;
  try
  {
    ExtractState st(w, h, PinholeCamera(fx, fy, cx, cy));
    st.income.setDevData(income_img);
    for (int i = 0; i < nframes; ++i)
    {
      auto *f = new DeviceImage<float>(w, h);
      f->setDevData(frames_img + (size_t)i * w * h);
      st.frames.push_back(f);
      FrameElement e;
      e.frame_ptr = f->dev_ptr;
      e.transform = se3_from(T_frame_income + 12 * i);
      st.mp.framelist_dev[i] = e;
    }
    DeviceImage<float> debug_image(w, h), depth_output(w, h);
    debug_image.setDevData(debug_inout);
    depth_output.zero();
    run_extract(st, nslots, debug_image, depth_output, levels_out, cost_out, msg_out);
    debug_image.getDevData(debug_inout);
    download(depth_output, dense_out);
  }
  catch (const std::exception &)
  {
    return 2;
  }
  return status();
}

// Depth fusion as SeedMatrix::fuse_output_depth does it.
//   depth_inout  w*h: upsampled depth in, fused depth (mu' or -1) out
//   seeds_inout  w*h*4 (a, b, mu, sigma^2): previous seeds in, new seeds out
//   T_income_last 12 floats, row-major 3x4 T_income<-lastfuse
//   table_out    w*h int (transform table after hole filling) or NULL
int qmref_fuse(int w, int h, float fx, float fy, float cx, float cy, float *depth_inout,
               float *seeds_inout, const float *T_income_last, int *table_out)
{
  try
  {
    PinholeCamera cam(fx, fy, cx, cy);
    DeviceImage<float> depth(w, h);
    DeviceImage<float4> seeds(w, h);
    DeviceImage<int> table(w, h);
    depth.setDevData(depth_inout);
    seeds.setDevData(reinterpret_cast<const float4 *>(seeds_inout));
    run_fuse(w, h, cam, depth, seeds, se3_from(T_income_last), &table);
    depth.getDevData(depth_inout);
    seeds.getDevData(reinterpret_cast<float4 *>(seeds_inout));
    download(table, table_out);
  }
  catch (const std::exception &)
  {
    return 2;
  }
  return status();
}

// Wall-clock time of the reference per-keyframe path (extract_depth then
// fuse_output_depth, with their per-frame allocations and synchronisations),
// iters timed repetitions after warmup untimed ones.  Returns ms per frame.
int qmref_time_frames(int w, int h, float fx, float fy, float cx, float cy,
                      const float *income_img, int nframes, const float *frames_img,
                      const float *T_frame_income, int nslots, const float *T_income_last,
                      int warmup, int iters, double *ms_per_frame)
{
  if (nframes < 1 || nframes > KEYFRAME_NUM || nslots < 1 || nslots > 10 ||
      DEPTH_NUM * nslots > 1024 || iters < 1)
    return 1;
  try
  {
    PinholeCamera cam(fx, fy, cx, cy);
    ExtractState st(w, h, cam);
    st.income.setDevData(income_img);
    for (int i = 0; i < nframes; ++i)
    {
      auto *f = new DeviceImage<float>(w, h);
      f->setDevData(frames_img + (size_t)i * w * h);
      st.frames.push_back(f);
      FrameElement e;
      e.frame_ptr = f->dev_ptr;
      e.transform = se3_from(T_frame_income + 12 * i);
      st.mp.framelist_dev[i] = e;
    }
    DeviceImage<float> debug_image(w, h), depth_output(w, h);
    DeviceImage<float4> seeds(w, h);
    seeds.zero();
    SE3<float> last = se3_from(T_income_last);
    double total = 0.0;
    for (int it = 0; it < warmup + iters; ++it)
    {
      cudaDeviceSynchronize();
      auto t0 = std::chrono::steady_clock::now();
      depth_output.zero();
      debug_image.zero();
      run_extract(st, nslots, debug_image, depth_output, nullptr, nullptr, nullptr);
      run_fuse(w, h, cam, depth_output, seeds, last, nullptr);
      cudaDeviceSynchronize();
      auto t1 = std::chrono::steady_clock::now();
      if (it >= warmup)
        total += std::chrono::duration<double, std::milli>(t1 - t0).count();
    }
    *ms_per_frame = total / iters;
  }
  catch (const std::exception &)
  {
    return 2;
  }
  return status();
}

__global__ void tex_sample_kernel(cudaTextureObject_t t, const float *uv, int n, float *out)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n)
    out[k] = tex2D<float>(t, uv[2 * k], uv[2 * k + 1]);
}

// Samples of a float image (w*h) through a texture object set up as the
// reference's bindTexture does (linear filtering, clamp, unnormalised
// coordinates) at n coordinates (x, y pairs).
int qmref_tex_sample(int w, int h, const float *img, const float *uv, int n, float *out)
{
  try
  {
    DeviceImage<float> image(w, h);
    image.setDevData(img);
    bindTexture(income_image_tex, image);
    const cudaTextureObject_t t = shim_live_textures()[(const void *)&income_image_tex];
    float *d_uv = nullptr, *d_out = nullptr;
    cudaMalloc(&d_uv, sizeof(float) * 2 * n);
    cudaMalloc(&d_out, sizeof(float) * n);
    cudaMemcpy(d_uv, uv, sizeof(float) * 2 * n, cudaMemcpyHostToDevice);
    tex_sample_kernel<<<(n + 255) / 256, 256>>>(t, d_uv, n, d_out);
    cudaMemcpy(out, d_out, sizeof(float) * n, cudaMemcpyDeviceToHost);
    cudaFree(d_uv);
    cudaFree(d_out);
    cudaUnbindTexture(income_image_tex);
  }
  catch (const std::exception &)
  {
    return 2;
  }
  return status();
}

// The semi-dense tracker as SeedMatrix::add_frames runs it, frame after
// frame: initial_keyframe (seed_matrix.cu:211-242) on the first frame, then
// update_keyframe (:401-446) and, when need_switchkeyframe (:198-209) says
// so, create_new_keyframe (:246-304) followed by set_income_as_keyframe.
//   frames       n*w*h float (values 0..255)
//   T_cur_world  n*12 floats (world -> camera)
//   debug_out    n*w*h: the debug image after each frame's update
//   seeds_out    w*h*8 floats or NULL: the seeds after the last frame,
//                (track_info x, y, z, 0, depth_info x, y, z, w) per pixel
//   modes_out    n ints: 1 first frame, 2 update, 3 update + keyframe switch
int qmref_semidense(int w, int h, float fx, float fy, float cx, float cy, int n,
                    const float *frames, const float *T_cur_world, float *debug_out,
                    float *seeds_out, int *modes_out)
{
  try
  {
    const float4 camera_para = make_float4(fx, cx, fy, cy);
    DeviceImage<float> income_image(w, h), keyframe_image(w, h), debug_image(w, h);
    DeviceImage<float2> income_gradient(w, h), keyframe_gradient(w, h);
    DeviceImage<DepthSeed> keyframe_semidense(w, h);
    keyframe_semidense.zero();
    income_gradient.zero();
    keyframe_gradient.zero();
    SE3<float> income_transform, keyframe_transform;
    dim3 block(8, 8), grid((w + 7) / 8, (h + 7) / 8);
    auto bind_all = [&]() {
      bindTexture(income_image_tex, income_image);
      bindTexture(income_gradient_tex, income_gradient);
      bindTexture(keyframe_image_tex, keyframe_image);
      bindTexture(keyframe_gradient_tex, keyframe_gradient);
    };
    auto unbind_all = [&]() {
      cudaUnbindTexture(income_image_tex);
      cudaUnbindTexture(income_gradient_tex);
      cudaUnbindTexture(keyframe_image_tex);
      cudaUnbindTexture(keyframe_gradient_tex);
    };
    for (int i = 0; i < n; ++i)
    {
      debug_image.zero();
      income_image.setDevData(frames + (size_t)i * w * h);
      income_transform = se3_from(T_cur_world + 12 * i);
      generate_gradient(income_image, income_gradient);
      cudaDeviceSynchronize();
      if (i == 0)
      {
        keyframe_image = income_image;
        keyframe_gradient = income_gradient;
        keyframe_transform = income_transform;
        bind_all();
        initialize_keyframe_kernel<<<grid, block>>>(keyframe_semidense.dev_ptr);
        cudaDeviceSynchronize();
        unbind_all();
        modes_out[i] = 1;
        debug_image.getDevData(debug_out + (size_t)i * w * h);
        continue;
      }
      bind_all();
      const SE3<float> key_to_income = income_transform * keyframe_transform.inv();
      update_keyframe_kernel<<<grid, block>>>(keyframe_semidense.dev_ptr, camera_para,
                                              key_to_income, debug_image.dev_ptr);
      regulizeDepth_FillHoles_kernel<<<grid, block>>>(keyframe_semidense.dev_ptr);
      regulizeDepth_kernel<<<grid, block>>>(keyframe_semidense.dev_ptr, false);
      depth_project_kernel<<<grid, block>>>(keyframe_semidense.dev_ptr, camera_para,
                                            key_to_income, debug_image.dev_ptr);
      cudaDeviceSynchronize();
      unbind_all();
      debug_image.getDevData(debug_out + (size_t)i * w * h);
      modes_out[i] = 2;
      // need_switchkeyframe
      const SE3<float> keyframe_pose = keyframe_transform.inv();
      const SE3<float> income_pose = income_transform.inv();
      const float3 kz = make_float3(keyframe_pose.data(0, 2), keyframe_pose.data(1, 2),
                                    keyframe_pose.data(2, 2));
      const float3 iz = make_float3(income_pose.data(0, 2), income_pose.data(1, 2),
                                    income_pose.data(2, 2));
      const float z_cos = dot(kz, iz);
      const float base_line =
          length(keyframe_pose.getTranslation() - income_pose.getTranslation());
      if (z_cos < 0.86 || base_line > 0.5)
      {
        bind_all();
        const SE3<float> old_to_new = income_transform * keyframe_transform.inv();
        DeviceImage<int> transform_table(w, h);
        DeviceImage<DepthSeed> new_keyframe(w, h);
        DeviceImage<float3> new_info(w, h);
        new_keyframe.zero();
        transform_table.zero();
        propogate_keyframe_kernel<<<grid, block>>>(keyframe_semidense.dev_ptr, camera_para,
                                                   old_to_new, transform_table.dev_ptr,
                                                   new_info.dev_ptr);
        cudaDeviceSynchronize();
        initialize_keyframe_kernel<<<grid, block>>>(new_keyframe.dev_ptr,
                                                    transform_table.dev_ptr, new_info.dev_ptr);
        cudaDeviceSynchronize();
        regulizeDepth_kernel<<<grid, block>>>(new_keyframe.dev_ptr, true);
        cudaDeviceSynchronize();
        regulizeDepth_FillHoles_kernel<<<grid, block>>>(new_keyframe.dev_ptr);
        cudaDeviceSynchronize();
        regulizeDepth_kernel<<<grid, block>>>(new_keyframe.dev_ptr, false);
        cudaDeviceSynchronize();
        keyframe_semidense = new_keyframe;
        unbind_all();
        keyframe_image = income_image;
        keyframe_gradient = income_gradient;
        keyframe_transform = income_transform;
        modes_out[i] = 3;
      }
    }
    if (seeds_out)
    {
      std::vector<DepthSeed> host((size_t)w * h);
      keyframe_semidense.getDevData(host.data());
      for (size_t o = 0; o < host.size(); ++o)
      {
        float *d = seeds_out + 8 * o;
        d[0] = host[o].track_info.x;
        d[1] = host[o].track_info.y;
        d[2] = host[o].track_info.z;
        d[3] = 0.0f;
        d[4] = host[o].depth_info.x;
        d[5] = host[o].depth_info.y;
        d[6] = host[o].depth_info.z;
        d[7] = host[o].depth_info.w;
      }
    }
  }
  catch (const std::exception &)
  {
    return 2;
  }
  return status();
}

} // extern "C"
