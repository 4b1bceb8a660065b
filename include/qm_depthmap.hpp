// C++ drop-in for quadmap::Depthmap (include/quadmap/depthmap.h:31-89 of
// open_quadtree_mapping) over the C-ABI of libqm_b200.so.
//
// Same constructor argument order (width, height, fx, cx, fy, cy, remap_1,
// remap_2, semi2dense_ratio), same add_frames / get* methods.  The cv::Mat
// overloads are compiled when QM_WITH_OPENCV is defined (the ROS node's
// build); raw-buffer overloads are always available.  Poses accept the
// reference's SE3<float> (anything with data[0..11] in row-major 3x4 order)
// or a float[12]; getT_world_ref() returns a QmPose, which converts
// implicitly to the reference's SE3<float>, so the publisher's
// `const quadmap::SE3<float> T_world_ref = depthmap_->getT_world_ref();`
// (publisher.cpp:138) compiles unchanged.  Errors from the library are
// thrown as quadmap::QmError (the reference throws quadmap::CudaException,
// cuda_exception.cuh:26-44).
#pragma once

#include <cstddef>
#include <cstdint>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "qm_capi.h"

#ifdef QM_WITH_OPENCV
#include <opencv2/imgproc/imgproc.hpp>
#endif

namespace quadmap
{

struct QmError : public std::runtime_error
{
  int status;
  QmError(int s, const std::string &what) : std::runtime_error(what), status(s) {}
};

inline void qm_check(int status)
{
  if (status != QM_OK)
    throw QmError(status, std::string("libqm_b200: ") + qm_last_error());
}

// A rigid transform as 12 floats, row-major 3x4 [R | t] (the layout of the
// reference's SE3<float>::data, se3.cuh).  Converts implicitly to any pose
// type whose `data` member takes data[0..11] = float, the reference's
// quadmap::SE3<float> among them.
struct QmPose
{
  float data[12];

  template <class SE3T, class = decltype(std::declval<SE3T &>().data[0] = 0.0f)>
  operator SE3T() const
  {
    SE3T s;
    for (int i = 0; i < 12; ++i)
      s.data[i] = data[i];
    return s;
  }
};

class Depthmap
{
public:
  Depthmap(size_t width, size_t height, float fx, float cx, float fy, float cy,
           int semi2dense_ratio = 1, const qm_params *params = nullptr, int device = 0)
      : width_(width), height_(height), fx_(fx), fy_(fy), cx_(cx), cy_(cy)
  {
    qm_check(qm_depthmap_create(&h_, (int)width, (int)height, fx, cx, fy, cy, semi2dense_ratio,
                                params, device));
    T_world_ref_[0] = T_world_ref_[5] = T_world_ref_[10] = 1.0f;
  }

#ifdef QM_WITH_OPENCV
  Depthmap(size_t width, size_t height, float fx, float cx, float fy, float cy, cv::Mat remap_1,
           cv::Mat remap_2, int semi2dense_ratio)
      : Depthmap(width, height, fx, cx, fy, cy, semi2dense_ratio)
  {
    remap_1_ = remap_1;
    remap_2_ = remap_2;
  }

  // Depthmap::add_frames (depthmap.h:46-47): undistorts on the host as
  // SeedMatrix::input_raw does (seed_matrix.cu:85), then runs the pipeline.
  template <class SE3T>
  bool add_frames(const cv::Mat &img_curr, const SE3T &T_curr_world)
  {
    cv::Mat und = img_curr;
    if (!remap_1_.empty())
      cv::remap(img_curr, und, remap_1_, remap_2_, cv::INTER_LINEAR, cv::BORDER_CONSTANT);
    float T[12];
    for (int i = 0; i < 12; ++i)
      T[i] = T_curr_world.data[i];
    const bool has = add_frames(und.data, und.step, T);
    if (has)
    {
      // fresh buffers per result, as SeedMatrix::get_result clones
      // (seed_matrix.cu:607-612): maps a caller still holds stay unchanged
      cv::Mat_<float> depth((int)height_, (int)width_), debug((int)height_, (int)width_);
      cv::Mat reference((int)height_, (int)width_, CV_8UC1);
      getDepthmap((float *)depth.data, depth.step / sizeof(float));
      getDebugmap((float *)debug.data, debug.step / sizeof(float));
      getReferenceImage(reference.data, reference.step);
      depth_out_ = depth;
      debug_out_ = debug;
      reference_out_ = reference;
    }
    return has;
  }
  const cv::Mat_<float> getDepthmap() const { return depth_out_; }
  const cv::Mat_<float> getDebugmap() const { return debug_out_; }
  const cv::Mat getReferenceImage() const { return reference_out_; }
#endif

  ~Depthmap()
  {
    if (h_)
      qm_depthmap_destroy(h_);
  }
  Depthmap(const Depthmap &) = delete;
  Depthmap &operator=(const Depthmap &) = delete;

  // Raw-buffer form: u8 image with row pitch `stride` bytes, world->camera pose.
  bool add_frames(const uint8_t *img, size_t stride, const float T_curr_world[12])
  {
    int has = 0;
    qm_check(qm_depthmap_add_frame(h_, img, stride, T_curr_world, &has));
    if (has)
      qm_check(qm_depthmap_get_T_world_ref(h_, T_world_ref_));
    return has != 0;
  }
  void getDepthmap(float *out, size_t stride) const
  {
    qm_check(qm_depthmap_get_depth(h_, out, stride));
  }
  void getDebugmap(float *out, size_t stride) const
  {
    qm_check(qm_depthmap_get_debug(h_, out, stride));
  }
  void getReferenceImage(uint8_t *out, size_t stride) const
  {
    qm_check(qm_depthmap_get_reference(h_, out, stride));
  }
  // Runs the semi-dense tracker on every frame (before the first frame), as
  // the reference's add_frames does; its depths seed the upsampler.
  void setSemidense(bool on) { qm_check(qm_depthmap_set_semidense(h_, on ? 1 : 0)); }
  // The cloud Publisher::publishPointCloud builds from the last result
  // (publisher.cpp:129-166): (x, y, z, intensity) per point, world frame.
  std::vector<float> getPointCloud() const
  {
    std::vector<float> pts((size_t)width_ * height_ * 4);
    int n = 0;
    qm_check(qm_depthmap_get_point_cloud(h_, pts.data(), (size_t)width_ * height_, &n));
    pts.resize((size_t)n * 4);
    return pts;
  }
  void getT_world_ref(float T[12]) const
  {
    for (int i = 0; i < 12; ++i)
      T[i] = T_world_ref_[i];
  }
  // getT_world_ref (depthmap.h:74): world <- reference frame of the last
  // result; assign it to the reference's SE3<float> directly.
  QmPose getT_world_ref() const
  {
    QmPose p;
    for (int i = 0; i < 12; ++i)
      p.data[i] = T_world_ref_[i];
    return p;
  }
  template <class SE3T>
  SE3T getT_world_ref() const
  {
    SE3T s;
    for (int i = 0; i < 12; ++i)
      s.data[i] = T_world_ref_[i];
    return s;
  }

  float getFx() const { return fx_; }
  float getFy() const { return fy_; }
  float getCx() const { return cx_; }
  float getCy() const { return cy_; }
  size_t getWidth() const { return width_; }
  size_t getHeight() const { return height_; }
  std::mutex &getRefImgMutex() { return ref_img_mutex_; }

private:
  qm_depthmap *h_ = nullptr;
  size_t width_, height_;
  float fx_, fy_, cx_, cy_;
  float T_world_ref_[12] = {};
  std::mutex ref_img_mutex_;
#ifdef QM_WITH_OPENCV
  cv::Mat remap_1_, remap_2_;
  cv::Mat_<float> depth_out_, debug_out_;
  cv::Mat reference_out_;
#endif
};

} // namespace quadmap
