// Camera streams: the frame-selection policy of SeedMatrix::add_frames
// (seed_matrix.cu:106-209) around the dense pipeline engine.
#pragma once

#include <deque>
#include <mutex>
#include <vector>

#include "engine.h"
#include "semidense.h"

namespace qm
{

// 3x4 row-major float rigid transform with the reference's SE3<float>
// arithmetic (se3.cuh:91-107 inverse, 179-195 composition).  The operation
// order is kept because the frame poses feed the cost projections, which
// are compared bit for bit with the reference.
struct SE3f
{
  float d[12];
  static SE3f identity();
  static SE3f from(const float *t12);
  SE3f inv() const;
};
SE3f operator*(const SE3f &l, const SE3f &r);

struct StreamDesc
{
  int W, H;
  Cam cam;
  int D, F;
  int ratio; // semi2dense_ratio
};

class StreamSet
{
public:
  StreamSet(int device, const qm_params &p, const std::vector<StreamDesc> &descs);
  ~StreamSet();

  int size() const { return (int)st_.size(); }
  // One frame per stream (imgs[i] host, pitch strides[i]); has_result out.
  // Waits for the results.
  void add_frames(const uint8_t *const *imgs, const size_t *strides, const float *T_curr_world,
                  int *has_result);
  // Pipelined form: runs the frame policy, enqueues the uploads, the dense
  // pipeline and (where depth_outs[i] is given) the download of stream i's
  // fused depth, and returns without waiting.  Up to two steps are in
  // flight: the uploads of step t+1 and the download of step t overlap the
  // pipeline.  Image buffers may be reused when the next submit (or wait)
  // returns; depth_outs are complete when wait() returns.
  void submit(const uint8_t *const *imgs, const size_t *strides, const float *T_curr_world,
              int *has_result, float *const *depth_outs, const size_t *depth_strides);
  // Waits for every submitted step.
  void wait();
  // Single-stream form used by the Depthmap facade.
  int add_frame(int i, const uint8_t *img, size_t stride, const float *T_curr_world);
  // Runs the semi-dense tracker on every frame of every stream, its
  // projected depths seeding the upsampler (as the reference's add_frames
  // does).  Only before the first frame.
  void set_semidense(bool on);
  bool semidense() const { return semidense_; }
  void run_resident();
  void profile_resident(float *ms, int *launches);

  void get_depth(int i, float *out, size_t stride);
  void get_debug(int i, float *out, size_t stride);
  // fused variance sigma^2 of every pixel of the last result
  void get_variance(int i, float *out, size_t stride);
  void get_reference(int i, uint8_t *out, size_t stride);
  // point cloud of the last result (Publisher::publishPointCloud,
  // publisher.cpp:129-166): up to `capacity` points of 4 floats (x, y, z,
  // intensity) into out; returns the number of points
  int get_point_cloud(int i, float *out, size_t capacity);
  // fused depth of several streams: all downloads enqueued, one wait
  void get_depths(const int *streams, int n, float *const *outs, const size_t *strides);
  void get_T_world_ref(int i, float *T) const;
  const StreamDesc &desc(int i) const { return st_[i].d; }
  const float *device_depth(int i) const
  {
    return eng_->buffers(i).dense[st_[i].out_parity];
  }
  Engine &engine() { return *eng_; }
  std::mutex &mutex() { return mu_; }

private:
  enum Outcome
  {
    kFirst,
    kSkip,
    kNoOutput,
    kOutput
  };
  struct RingFrame
  {
    int slot;
    SE3f T; // T_frame<-world
  };
  struct State
  {
    StreamDesc d;
    uint8_t *pool = nullptr; // (ring capacity + 2) frames, dense W x H
    std::vector<int> free_slots;
    std::deque<RingFrame> ring;
    int income_slot = -1;
    SE3f income_T, keyframe_T, fuse_T;
    int frame_index = 0;
    bool initialized = false;
    Outcome outcome = kSkip;
    bool has_ref = false; // the pool's last slot holds the last result's image
    int out_parity = 0;   // output buffer of the last result
    SE3f T_world_ref;
    // semi-dense tracker: float images (keyframe / incoming, roles swap on a
    // keyframe switch) with their texture views, seeds (two buffers each of
    // trk and dep), and this frame's step
    float *sd_img[2] = {nullptr, nullptr};
    cudaTextureObject_t sd_tex[2] = {0, 0};
    size_t sd_pitch = 0;
    float4 *sd_trk[2] = {nullptr, nullptr}, *sd_dep[2] = {nullptr, nullptr};
    int sd_key = 0; // sd_img index of the keyframe
    int sd_mode = kSdNone;
    SE3f sd_T;      // T_income<-key of this frame's step
  };

  Outcome begin_frame(int i, const uint8_t *img, size_t stride, const float *T);
  void end_frame(int i, int parity);
  // one step of the streams in `which` (see submit)
  void step(const std::vector<int> &which, const uint8_t *const *imgs, const size_t *strides,
            const float *T_curr_world, int *has_result, float *const *depth_outs,
            const size_t *depth_strides);
  // waits for the step of parity p and recycles the frame slots it freed
  void retire(int p);
  bool need_add_reference(const State &s) const;
  bool need_switch_keyframe(const State &s) const;
  uint8_t *frame_ptr(const State &s, int slot) const
  {
    return s.pool + (size_t)slot * s.d.W * s.d.H;
  }
  uint8_t *ref_ptr(const State &s) const { return frame_ptr(s, QM_RING_CAPACITY + 2); }
  void keep_reference(State &s);
  // enqueues the semi-dense step of the streams in `which` on the engine
  // stream (after their uploads)
  void semidense_step(const std::vector<int> &which, int parity);

  int device_;
  std::vector<State> st_;
  std::unique_ptr<Engine> eng_;
  std::vector<int> last_active_;
  std::mutex mu_;
  // pipelining: uploads and downloads run on their own streams; per step
  // parity, events mark the end of its uploads, of its pipeline and of its
  // downloads, and the frame slots it freed wait in `pending_` until then
  cudaStream_t up_ = nullptr, down_ = nullptr;
  cudaEvent_t ev_up_[2] = {}, ev_comp_[2] = {}, ev_done_[2] = {};
  std::vector<std::pair<int, int>> pending_[2]; // (stream, slot)
  bool inflight_[2] = {false, false};
  long step_ = 0;
  void *pc_buf_ = nullptr; // point-cloud staging (first get_point_cloud)
  size_t pc_bytes_ = 0;
  bool semidense_ = false;
  bool started_ = false; // a frame has been added
  // semi-dense job tables: pinned per parity, one device copy
  SdJob *h_sdjobs_[2] = {nullptr, nullptr};
  int *h_sdprefix_[2] = {nullptr, nullptr};
  SdJob *d_sdjobs_ = nullptr;
  int *d_sdprefix_ = nullptr;
};

} // namespace qm
