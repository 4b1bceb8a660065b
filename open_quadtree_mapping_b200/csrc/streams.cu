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
  for (auto &s : st_)
    if (s.pool)
      cudaFree(s.pool);
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
  check(cudaMemcpy2DAsync(frame_ptr(s, s.income_slot), W, img, stride, W, H,
                          cudaMemcpyHostToDevice, eng_->stream()),
        "image upload");
  s.income_T = SE3f::from(T);
  if (!s.initialized)
  {
    s.keyframe_T = s.income_T;
    s.initialized = true;
    return kFirst;
  }
  // The keyframe switch only matters to the semi-dense tracker; the pose is
  // kept so that the stream state mirrors the reference's.
  if (need_switch_keyframe(s))
    s.keyframe_T = s.income_T;
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

void StreamSet::end_frame(int i)
{
  State &s = st_[i];
  const size_t P = (size_t)s.d.W * s.d.H;
  bool keep_income = false;
  if (s.outcome == kFirst)
  {
    const JobBuffers &b = eng_->buffers(i);
    check(cudaMemsetAsync(b.dense, 0, P * sizeof(float), eng_->stream()), "memset");
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
        s.free_slots.push_back(s.ring.back().slot);
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
  if (!keep_income)
    s.free_slots.push_back(s.income_slot);
  s.income_slot = -1;
}

void StreamSet::add_frames(const uint8_t *const *imgs, const size_t *strides,
                           const float *T_curr_world, int *has_result)
{
  check(cudaSetDevice(device_), "cudaSetDevice");
  std::vector<int> active;
  for (int i = 0; i < size(); ++i)
  {
    st_[i].outcome = begin_frame(i, imgs[i], strides[i], T_curr_world + 12 * i);
    if (st_[i].outcome == kOutput)
      active.push_back(i);
  }
  if (!active.empty())
  {
    eng_->run(active);
    last_active_ = active;
  }
  for (int i = 0; i < size(); ++i)
  {
    end_frame(i);
    has_result[i] = (st_[i].outcome == kFirst || st_[i].outcome == kOutput) ? 1 : 0;
  }
  check(cudaStreamSynchronize(eng_->stream()), "frame");
}

int StreamSet::add_frame(int i, const uint8_t *img, size_t stride, const float *T_curr_world)
{
  check(cudaSetDevice(device_), "cudaSetDevice");
  st_[i].outcome = begin_frame(i, img, stride, T_curr_world);
  if (st_[i].outcome == kOutput)
  {
    eng_->run({i});
    last_active_ = {i};
  }
  end_frame(i);
  check(cudaStreamSynchronize(eng_->stream()), "frame");
  return (st_[i].outcome == kFirst || st_[i].outcome == kOutput) ? 1 : 0;
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
  eng_->run(all);
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
  const State &s = st_[i];
  check(cudaMemcpy2D(out, stride * sizeof(float), eng_->buffers(i).dense, s.d.W * sizeof(float),
                     s.d.W * sizeof(float), s.d.H, cudaMemcpyDeviceToHost),
        "depth download");
}

void StreamSet::get_debug(int i, float *out, size_t stride)
{
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
  for (int k = 0; k < n; ++k)
  {
    const State &s = st_[streams[k]];
    check(cudaMemcpy2DAsync(outs[k], strides[k] * sizeof(float), eng_->buffers(streams[k]).dense,
                            s.d.W * sizeof(float), s.d.W * sizeof(float), s.d.H,
                            cudaMemcpyDeviceToHost, eng_->stream()),
          "depth download");
  }
  check(cudaStreamSynchronize(eng_->stream()), "depth download");
}

void StreamSet::get_reference(int i, uint8_t *out, size_t stride)
{
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
