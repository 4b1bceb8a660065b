// Camera streams around the dense pipeline (see streams.h).
//
// Frame policy, after SeedMatrix::add_frames (seed_matrix.cu:106-169):
//  * frame 1 initialises the stream and reports a (zero) result
//    (seed_matrix.cu:122-128);
//  * frames whose index is not a multiple of semi2dense_ratio report nothing
//    (seed_matrix.cu:144-145);
//  * otherwise, when the reference-frame ring holds more than 10 frames, the
//    dense pipeline runs on the current frame (seed_matrix.cu:151-155), the
//    current frame joins the ring front when it moved enough
//    (need_add_reference, seed_matrix.cu:171-198; capacity 60), and the depth
//    is fused with the previous result (seed_matrix.cu:163-167).
// Measurement slot f reads ring frame floor(0.9 f) (the reference's zeroed
// pixel-age table, depth_extract.cu:153-166) with pose
// T_frame<-world * T_income<-world^-1 (seed_matrix.cu:457-464).
// Frames live in a per-stream device pool; joining the ring hands the slot
// over instead of copying the image.
#include "streams.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace qm
{

SE3f SE3f::identity()
{
  SE3f s;
  std::memset(s.d, 0, sizeof(s.d));
  s.d[0] = s.d[5] = s.d[10] = 1.0f;
  return s;
}

SE3f SE3f::from(const float *t)
{
  SE3f s;
  std::memcpy(s.d, t, sizeof(s.d));
  return s;
}

SE3f SE3f::inv() const
{
  SE3f r = SE3f::identity();
  const float *a = d;
  r.d[0] = a[0];
  r.d[1] = a[4];
  r.d[2] = a[8];
  r.d[4] = a[1];
  r.d[5] = a[5];
  r.d[6] = a[9];
  r.d[8] = a[2];
  r.d[9] = a[6];
  r.d[10] = a[10];
  r.d[3] = -a[0] * a[3] - a[4] * a[7] - a[8] * a[11];
  r.d[7] = -a[1] * a[3] - a[5] * a[7] - a[9] * a[11];
  r.d[11] = -a[2] * a[3] - a[6] * a[7] - a[10] * a[11];
  return r;
}

SE3f operator*(const SE3f &lhs, const SE3f &rhs)
{
  const float *l = lhs.d, *r = rhs.d;
  SE3f o;
  for (int row = 0; row < 3; ++row)
  {
    const float *a = l + 4 * row;
    for (int c = 0; c < 3; ++c)
      o.d[4 * row + c] = a[0] * r[c] + a[1] * r[4 + c] + a[2] * r[8 + c];
    o.d[4 * row + 3] = a[3] + a[0] * r[3] + a[1] * r[7] + a[2] * r[11];
  }
  return o;
}

namespace
{
constexpr int kRing = QM_RING_CAPACITY;

float dot3(const float *a, const float *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// z axis of the camera in world coordinates and the camera centre, from the
// camera->world pose (the reference reads data(0..2, 2) and the translation)
void axis_and_centre(const SE3f &T_world_cam, float z[3], float c[3])
{
  z[0] = T_world_cam.d[2];
  z[1] = T_world_cam.d[6];
  z[2] = T_world_cam.d[10];
  c[0] = T_world_cam.d[3];
  c[1] = T_world_cam.d[7];
  c[2] = T_world_cam.d[11];
}

bool moved(const SE3f &a_cam_world, const SE3f &b_cam_world, double min_cos, double max_base)
{
  const SE3f a = a_cam_world.inv(), b = b_cam_world.inv();
  float za[3], ca[3], zb[3], cb[3];
  axis_and_centre(a, za, ca);
  axis_and_centre(b, zb, cb);
  const float z_cos = dot3(za, zb);
  const float dv[3] = {ca[0] - cb[0], ca[1] - cb[1], ca[2] - cb[2]};
  const float base = std::sqrt(dot3(dv, dv));
  return (z_cos < min_cos || base > max_base);
}
} // namespace

StreamSet::StreamSet(int device, const qm_params &p, const std::vector<StreamDesc> &descs)
    : device_(device)
{
  std::vector<Shape> shapes;
  for (const auto &d : descs)
  {
    if (d.ratio < 1)
      throw CudaError{QM_ERR_INVALID_ARG, "semi2dense_ratio must be >= 1"};
    shapes.push_back(Shape{d.W, d.H, d.D, d.F, d.cam});
  }
  eng_ = std::make_unique<Engine>(device, p, shapes);
  check(cudaStreamCreateWithFlags(&up_, cudaStreamNonBlocking), "cudaStreamCreate");
  check(cudaStreamCreateWithFlags(&down_, cudaStreamNonBlocking), "cudaStreamCreate");
  for (int q = 0; q < 2; ++q)
  {
    check(cudaEventCreateWithFlags(&ev_up_[q], cudaEventDisableTiming), "cudaEventCreate");
    check(cudaEventCreateWithFlags(&ev_comp_[q], cudaEventDisableTiming), "cudaEventCreate");
    check(cudaEventCreateWithFlags(&ev_done_[q], cudaEventDisableTiming), "cudaEventCreate");
  }
  st_.resize(descs.size());
  for (size_t i = 0; i < descs.size(); ++i)
  {
    State &s = st_[i];
    s.d = descs[i];
    const size_t frame = (size_t)s.d.W * s.d.H;
    // ring + income + spare frames, and the image of the last result
    check(cudaMalloc((void **)&s.pool, frame * (kRing + 3)), "frame pool allocation");
    for (int k = kRing + 1; k >= 0; --k)
      s.free_slots.push_back(k);
    s.income_T = s.keyframe_T = s.fuse_T = s.T_world_ref = SE3f::identity();
  }
}

StreamSet::~StreamSet()
{
  cudaSetDevice(device_);
  if (up_)
    cudaStreamSynchronize(up_);
  if (down_)
    cudaStreamSynchronize(down_);
  cudaStreamSynchronize(eng_->stream());
  for (int q = 0; q < 2; ++q)
  {
    if (ev_up_[q])
      cudaEventDestroy(ev_up_[q]);
    if (ev_comp_[q])
      cudaEventDestroy(ev_comp_[q]);
    if (ev_done_[q])
      cudaEventDestroy(ev_done_[q]);
  }
  if (up_)
    cudaStreamDestroy(up_);
  if (down_)
    cudaStreamDestroy(down_);
  for (auto &s : st_)
    if (s.pool)
      cudaFree(s.pool);
  if (pc_buf_)
    cudaFree(pc_buf_);
  for (auto &s : st_)
    for (int k = 0; k < 2; ++k)
    {
      if (s.sd_tex[k])
        cudaDestroyTextureObject(s.sd_tex[k]);
      if (s.sd_img[k])
        cudaFree(s.sd_img[k]);
      if (s.sd_trk[k])
        cudaFree(s.sd_trk[k]);
      if (s.sd_dep[k])
        cudaFree(s.sd_dep[k]);
    }
  for (int q = 0; q < 2; ++q)
  {
    if (h_sdjobs_[q])
      cudaFreeHost(h_sdjobs_[q]);
    if (h_sdprefix_[q])
      cudaFreeHost(h_sdprefix_[q]);
  }
  if (d_sdjobs_)
    cudaFree(d_sdjobs_);
  if (d_sdprefix_)
    cudaFree(d_sdprefix_);
}

void StreamSet::set_semidense(bool on)
{
  if (on == semidense_)
    return;
  if (started_)
    throw CudaError{QM_ERR_STATE, "the semi-dense tracker is switched before the first frame"};
  check(cudaSetDevice(device_), "cudaSetDevice");
  if (on && !d_sdjobs_)
  {
    const int n = size();
    for (auto &s : st_)
    {
      const size_t P = (size_t)s.d.W * s.d.H;
      s.sd_pitch = sd_texture_pitch(s.d.W);
      for (int k = 0; k < 2; ++k)
      {
        check(cudaMalloc((void **)&s.sd_img[k], s.sd_pitch * s.d.H * sizeof(float)),
              "semi-dense image allocation");
        check(cudaMalloc((void **)&s.sd_trk[k], P * sizeof(float4)), "seed allocation");
        check(cudaMalloc((void **)&s.sd_dep[k], P * sizeof(float4)), "seed allocation");
        check(cudaMemset(s.sd_img[k], 0, s.sd_pitch * s.d.H * sizeof(float)), "memset");
        check(cudaMemset(s.sd_trk[k], 0, P * sizeof(float4)), "memset");
        check(cudaMemset(s.sd_dep[k], 0, P * sizeof(float4)), "memset");
        s.sd_tex[k] = sd_make_texture(s.sd_img[k], s.d.W, s.d.H, s.sd_pitch);
        if (!s.sd_tex[k])
          throw CudaError{QM_ERR_CUDA, "texture object creation failed"};
      }
    }
    for (int q = 0; q < 2; ++q)
    {
      check(cudaHostAlloc((void **)&h_sdjobs_[q], sizeof(SdJob) * n, cudaHostAllocDefault),
            "pinned allocation");
      check(cudaHostAlloc((void **)&h_sdprefix_[q], sizeof(int) * (n + 1), cudaHostAllocDefault),
            "pinned allocation");
    }
    check(cudaMalloc((void **)&d_sdjobs_, sizeof(SdJob) * n), "device allocation");
    check(cudaMalloc((void **)&d_sdprefix_, sizeof(int) * (n + 1)), "device allocation");
  }
  semidense_ = on;
  eng_->set_keep_sparse(on);
}

void StreamSet::semidense_step(const std::vector<int> &which, int parity)
{
  SdJob *jobs = h_sdjobs_[parity];
  int *prefix = h_sdprefix_[parity];
  const bool ieee = eng_->params().arith == QM_ARITH_IEEE;
  int n = 0;
  prefix[0] = 0;
  for (int i : which)
  {
    State &s = st_[i];
    SdJob &J = jobs[n];
    std::memset(&J, 0, sizeof(J));
    J.W = s.d.W;
    J.H = s.d.H;
    J.fx = s.d.cam.fx;
    J.fy = s.d.cam.fy;
    J.cx = s.d.cam.cx;
    J.cy = s.d.cam.cy;
    J.mode = s.sd_mode;
    J.inc = frame_ptr(s, s.income_slot);
    J.inc_f = s.sd_img[s.sd_key ^ 1];
    J.key_f = s.sd_img[s.sd_key];
    J.pitch = s.sd_pitch;
    J.inc_tex = ieee ? 0 : s.sd_tex[s.sd_key ^ 1];
    J.key_tex = ieee ? 0 : s.sd_tex[s.sd_key];
    for (int k = 0; k < 2; ++k)
    {
      J.trk[k] = s.sd_trk[k];
      J.dep[k] = s.sd_dep[k];
    }
    J.cur = 0;
    J.debug = eng_->buffers(i).sparse;
    J.zkey = eng_->buffers(i).sdkey;
    std::memcpy(J.T, s.sd_T.d, sizeof(J.T));
    prefix[n + 1] = prefix[n] + sd_blocks(s.d.W, s.d.H);
    ++n;
    // the incoming image becomes the keyframe after a first frame or a switch
    if (s.sd_mode == kSdInit || s.sd_mode == kSdSwitch)
      s.sd_key ^= 1;
  }
  if (n == 0)
    return;
  const cudaStream_t cs = eng_->stream();
  check(cudaMemcpyAsync(d_sdjobs_, jobs, sizeof(SdJob) * n, cudaMemcpyHostToDevice, cs),
        "semi-dense job upload");
  check(cudaMemcpyAsync(d_sdprefix_, prefix, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, cs),
        "semi-dense job upload");
  SdBatch B;
  std::memset(&B, 0, sizeof(B));
  B.jobs = d_sdjobs_;
  B.prefix = d_sdprefix_;
  B.njobs = n;
  launch_semidense(B, prefix[n], ieee ? 1 : 0, cs);
  check(cudaGetLastError(), "semi-dense launch");
}

bool StreamSet::need_add_reference(const State &s) const
{
  if (s.ring.empty())
    return true;
  return moved(s.ring.front().T, s.income_T, 0.95, 0.03);
}

bool StreamSet::need_switch_keyframe(const State &s) const
{
  return moved(s.keyframe_T, s.income_T, 0.86, 0.5);
}

StreamSet::Outcome StreamSet::begin_frame(int i, const uint8_t *img, size_t stride,
                                          const float *T)
{
  State &s = st_[i];
  const int W = s.d.W, H = s.d.H;
  if (!img || !T || stride < (size_t)W)
    throw CudaError{QM_ERR_INVALID_ARG, "image pointer, stride or pose invalid"};
  s.frame_index++;
  s.income_slot = s.free_slots.back();
  s.free_slots.pop_back();
  // a dense image goes up as one linear copy (row-by-row 2D copies of short
  // rows are much slower on the copy engines)
  if (stride == (size_t)W)
    check(cudaMemcpyAsync(frame_ptr(s, s.income_slot), img, (size_t)W * H,
                          cudaMemcpyHostToDevice, up_),
          "image upload");
  else
    check(cudaMemcpy2DAsync(frame_ptr(s, s.income_slot), W, img, stride, W, H,
                            cudaMemcpyHostToDevice, up_),
          "image upload");
  s.income_T = SE3f::from(T);
  if (!s.initialized)
  {
    s.keyframe_T = s.income_T;
    s.initialized = true;
    s.sd_mode = kSdInit;
    s.sd_T = SE3f::identity();
    return kFirst;
  }
  // the semi-dense step updates the seeds against the current keyframe
  // (key_to_income, seed_matrix.cu:417) and then, when the camera moved far
  // enough, makes this frame the keyframe (seed_matrix.cu:131-140)
  s.sd_T = s.income_T * s.keyframe_T.inv();
  s.sd_mode = kSdUpdate;
  if (need_switch_keyframe(s))
  {
    s.keyframe_T = s.income_T;
    s.sd_mode = kSdSwitch;
  }
  if (s.frame_index % s.d.ratio != 0)
    return kSkip;
  if ((int)s.ring.size() <= 10)
    return kNoOutput;
  std::vector<const uint8_t *> slots(s.d.F);
  std::vector<float> Ts(12 * s.d.F);
  const SE3f income_inv = s.income_T.inv();
  for (int f = 0; f < s.d.F; ++f)
  {
    int k = (int)((float)9 / 10.0 * (float)f);
    if (k >= (int)s.ring.size())
      k = (int)s.ring.size() - 1;
    const RingFrame &rf = s.ring[k];
    slots[f] = frame_ptr(s, rf.slot);
    const SE3f T_slot = rf.T * income_inv;
    std::memcpy(Ts.data() + 12 * f, T_slot.d, sizeof(T_slot.d));
  }
  const SE3f T_fuse = s.income_T * s.fuse_T.inv();
  eng_->set_inputs(i, frame_ptr(s, s.income_slot), W, slots.data(), W, Ts.data(), T_fuse.d);
  return kOutput;
}

// The image of the last result stays on the device (a copy into the pool's
// last slot, ordered after the frame's upload on the engine stream) and is
// only downloaded when asked for.
void StreamSet::keep_reference(State &s)
{
  check(cudaMemcpyAsync(ref_ptr(s), frame_ptr(s, s.income_slot), (size_t)s.d.W * s.d.H,
                        cudaMemcpyDeviceToDevice, eng_->stream()),
        "reference image copy");
  s.has_ref = true;
}

void StreamSet::end_frame(int i, int parity)
{
  State &s = st_[i];
  const size_t P = (size_t)s.d.W * s.d.H;
  bool keep_income = false;
  if (s.outcome == kFirst)
  {
    const JobBuffers &b = eng_->buffers(i);
    check(cudaMemsetAsync(eng_->dense(i), 0, P * sizeof(float), eng_->stream()), "memset");
    check(cudaMemsetAsync(b.sparse, 0, P * sizeof(float), eng_->stream()), "memset");
    keep_reference(s);
    s.T_world_ref = s.income_T.inv();
  }
  else if (s.outcome == kNoOutput || s.outcome == kOutput)
  {
    if (need_add_reference(s))
    {
      s.ring.push_front(RingFrame{s.income_slot, s.income_T});
      keep_income = true;
      if ((int)s.ring.size() > kRing)
      {
        pending_[parity].push_back({i, s.ring.back().slot});
        s.ring.pop_back();
      }
    }
    if (s.outcome == kOutput)
    {
      s.fuse_T = s.income_T;
      keep_reference(s);
      s.T_world_ref = s.income_T.inv();
    }
  }
  // a freed slot may still be read by this step's pipeline: it becomes free
  // again once the step has retired
  if (!keep_income)
    pending_[parity].push_back({i, s.income_slot});
  s.income_slot = -1;
}

void StreamSet::retire(int p)
{
  if (!inflight_[p])
    return;
  check(cudaEventSynchronize(ev_done_[p]), "step");
  for (const auto &f : pending_[p])
    st_[f.first].free_slots.push_back(f.second);
  pending_[p].clear();
  inflight_[p] = false;
}

void StreamSet::wait()
{
  // the older step first, so slots return in the order they were freed
  const int p = (int)(step_ & 1);
  retire(p);
  retire(p ^ 1);
}

void StreamSet::step(const std::vector<int> &which, const uint8_t *const *imgs,
                     const size_t *strides, const float *T_curr_world, int *has_result,
                     float *const *depth_outs, const size_t *depth_strides)
{
  // every argument is checked before any stream's state changes, so a
  // rejected call leaves the set as it was and launches nothing: the cost
  // kernel gathers measurement pixels without clamping and relies on poses
  // that keep projections finite
  for (size_t k = 0; k < which.size(); ++k)
  {
    const int i = which[k];
    if (!imgs[k] || strides[k] < (size_t)st_[i].d.W)
      throw CudaError{QM_ERR_INVALID_ARG, "image pointer or stride invalid"};
    if (!rigid_enough(T_curr_world + 12 * k))
      throw CudaError{QM_ERR_INVALID_ARG,
                      "frame pose is not a rigid transform (finite, rotation rows bounded)"};
  }
  check(cudaSetDevice(device_), "cudaSetDevice");
  const int p = (int)(step_ & 1);
  // step t-2 (same parity) must be done: its output buffer, pinned tables
  // and freed slots are reused now; step t-1's uploads must be done so that
  // the caller may reuse its image buffers
  retire(p);
  if (inflight_[p ^ 1])
    check(cudaEventSynchronize(ev_up_[p ^ 1]), "upload");
  eng_->set_parity(p);
  started_ = true;
  std::vector<int> active;
  for (size_t k = 0; k < which.size(); ++k)
  {
    const int i = which[k];
    st_[i].outcome = begin_frame(i, imgs[k], strides[k], T_curr_world + 12 * k);
    if (st_[i].outcome == kOutput)
      active.push_back(i);
  }
  check(cudaEventRecord(ev_up_[p], up_), "event");
  check(cudaStreamWaitEvent(eng_->stream(), ev_up_[p], 0), "event wait");
  if (semidense_)
    semidense_step(which, p);
  if (!active.empty())
  {
    eng_->launch(active);
    last_active_ = active;
  }
  for (size_t k = 0; k < which.size(); ++k)
  {
    end_frame(which[k], p);
    const Outcome o = st_[which[k]].outcome;
    has_result[k] = (o == kFirst || o == kOutput) ? 1 : 0;
    if (has_result[k])
      st_[which[k]].out_parity = p;
  }
  check(cudaEventRecord(ev_comp_[p], eng_->stream()), "event");
  check(cudaStreamWaitEvent(down_, ev_comp_[p], 0), "event wait");
  if (depth_outs)
    for (size_t k = 0; k < which.size(); ++k)
    {
      if (!has_result[k] || !depth_outs[k])
        continue;
      const State &s = st_[which[k]];
      const float *src = eng_->dense(which[k]);
      const size_t stride = depth_strides ? depth_strides[k] : (size_t)s.d.W;
      if (stride == (size_t)s.d.W)
        check(cudaMemcpyAsync(depth_outs[k], src, sizeof(float) * s.d.W * s.d.H,
                              cudaMemcpyDeviceToHost, down_),
              "depth download");
      else
        check(cudaMemcpy2DAsync(depth_outs[k], stride * sizeof(float), src,
                                s.d.W * sizeof(float), s.d.W * sizeof(float), s.d.H,
                                cudaMemcpyDeviceToHost, down_),
              "depth download");
    }
  check(cudaEventRecord(ev_done_[p], down_), "event");
  inflight_[p] = true;
  ++step_;
}

void StreamSet::submit(const uint8_t *const *imgs, const size_t *strides,
                       const float *T_curr_world, int *has_result, float *const *depth_outs,
                       const size_t *depth_strides)
{
  if (depth_outs)
    for (int i = 0; i < size(); ++i)
      if (depth_outs[i] && depth_strides && depth_strides[i] < (size_t)st_[i].d.W)
        throw CudaError{QM_ERR_INVALID_ARG, "depth stride smaller than the width"};
  std::vector<int> all(size());
  for (int i = 0; i < size(); ++i)
    all[i] = i;
  step(all, imgs, strides, T_curr_world, has_result, depth_outs, depth_strides);
}

void StreamSet::add_frames(const uint8_t *const *imgs, const size_t *strides,
                           const float *T_curr_world, int *has_result)
{
  submit(imgs, strides, T_curr_world, has_result, nullptr, nullptr);
  wait();
}

int StreamSet::add_frame(int i, const uint8_t *img, size_t stride, const float *T_curr_world)
{
  int has = 0;
  step({i}, &img, &stride, T_curr_world, &has, nullptr, nullptr);
  wait();
  return has;
}

void StreamSet::run_resident()
{
  if (last_active_.empty())
    throw CudaError{QM_ERR_STATE, "no dense run has happened yet"};
  std::vector<int> all;
  for (int i = 0; i < size(); ++i)
    all.push_back(i);
  if (last_active_ != all)
    throw CudaError{QM_ERR_STATE, "every stream must have produced a depth map once"};
  wait();
  eng_->run(all);
  for (auto &s : st_)
    s.out_parity = eng_->parity();
}

void StreamSet::profile_resident(float *ms, int *launches)
{
  run_resident(); // validates the state (and warms the plan)
  std::vector<int> all;
  for (int i = 0; i < size(); ++i)
    all.push_back(i);
  eng_->profile(all, ms, launches);
}

void StreamSet::get_depth(int i, float *out, size_t stride)
{
  wait();
  const State &s = st_[i];
  check(cudaMemcpy2D(out, stride * sizeof(float), device_depth(i), s.d.W * sizeof(float),
                     s.d.W * sizeof(float), s.d.H, cudaMemcpyDeviceToHost),
        "depth download");
}

void StreamSet::get_variance(int i, float *out, size_t stride)
{
  wait();
  const State &s = st_[i];
  const size_t P = (size_t)s.d.W * s.d.H;
  // the row-pass buffer is idle between runs: stage the variances there
  float *tmp = reinterpret_cast<float *>(eng_->buffers(i).rowres);
  launch_seed_variance(eng_->seeds(i), tmp, (long)P, eng_->stream());
  check(cudaGetLastError(), "variance extraction");
  check(cudaMemcpy2DAsync(out, stride * sizeof(float), tmp, s.d.W * sizeof(float),
                          s.d.W * sizeof(float), s.d.H, cudaMemcpyDeviceToHost, eng_->stream()),
        "variance download");
  check(cudaStreamSynchronize(eng_->stream()), "variance download");
}

int StreamSet::get_point_cloud(int i, float *out, size_t capacity)
{
  wait();
  const State &s = st_[i];
  if (!s.has_ref)
    throw CudaError{QM_ERR_STATE, "no result yet"};
  const int W = s.d.W, H = s.d.H;
  // one device buffer for every stream: points of the largest image, the
  // count and the scan workspace (allocated on the first call)
  size_t need = 0;
  for (const auto &t : st_)
    need = std::max(need, (size_t)t.d.W * t.d.H * sizeof(float4) + 256 +
                              point_cloud_workspace(t.d.W, t.d.H));
  if (!pc_buf_)
  {
    check(cudaMalloc(&pc_buf_, need), "point-cloud buffer");
    pc_bytes_ = need;
  }
  float4 *pts = reinterpret_cast<float4 *>(pc_buf_);
  char *tail = reinterpret_cast<char *>(pc_buf_) + (((size_t)W * H * sizeof(float4) + 255) & ~size_t(255));
  int *d_count = reinterpret_cast<int *>(tail);
  void *ws = tail + 256;
  launch_point_cloud(device_depth(i), (size_t)W, ref_ptr(s), (size_t)W, W, H, s.d.cam,
                     s.T_world_ref.d, pts, d_count, ws, eng_->stream());
  check(cudaGetLastError(), "point cloud");
  int n = 0;
  check(cudaMemcpyAsync(&n, d_count, sizeof(int), cudaMemcpyDeviceToHost, eng_->stream()),
        "point count");
  check(cudaStreamSynchronize(eng_->stream()), "point cloud");
  const size_t take = std::min((size_t)n, capacity);
  if (take > 0)
    check(cudaMemcpy(out, pts, take * sizeof(float4), cudaMemcpyDeviceToHost), "point download");
  return n;
}

void StreamSet::get_debug(int i, float *out, size_t stride)
{
  wait();
  const State &s = st_[i];
  check(cudaMemcpy2D(out, stride * sizeof(float), eng_->buffers(i).sparse, s.d.W * sizeof(float),
                     s.d.W * sizeof(float), s.d.H, cudaMemcpyDeviceToHost),
        "debug download");
}

void StreamSet::get_depths(const int *streams, int n, float *const *outs, const size_t *strides)
{
  for (int k = 0; k < n; ++k)
    if (streams[k] < 0 || streams[k] >= size() || !outs[k] || strides[k] < (size_t)st_[streams[k]].d.W)
      throw CudaError{QM_ERR_INVALID_ARG, "bad stream index, output pointer or stride"};
  wait();
  for (int k = 0; k < n; ++k)
  {
    const State &s = st_[streams[k]];
    const float *src = device_depth(streams[k]);
    if (strides[k] == (size_t)s.d.W)
      check(cudaMemcpyAsync(outs[k], src, sizeof(float) * s.d.W * s.d.H, cudaMemcpyDeviceToHost,
                            eng_->stream()),
            "depth download");
    else
      check(cudaMemcpy2DAsync(outs[k], strides[k] * sizeof(float), src, s.d.W * sizeof(float),
                              s.d.W * sizeof(float), s.d.H, cudaMemcpyDeviceToHost,
                              eng_->stream()),
            "depth download");
  }
  check(cudaStreamSynchronize(eng_->stream()), "depth download");
}

void StreamSet::get_reference(int i, uint8_t *out, size_t stride)
{
  wait();
  const State &s = st_[i];
  if (!s.has_ref)
    throw CudaError{QM_ERR_STATE, "no result yet"};
  check(cudaMemcpy2D(out, stride, ref_ptr(s), s.d.W, s.d.W, s.d.H, cudaMemcpyDeviceToHost),
        "reference download");
}

void StreamSet::get_T_world_ref(int i, float *T) const
{
  std::memcpy(T, st_[i].T_world_ref.d, 12 * sizeof(float));
}

} // namespace qm
