// The reference's own callers of quadmap::Depthmap, as call shapes: the ROS
// node's construction and frame callback (depthmap_node.cpp:95, 120-139)
// and the publisher's reads (publisher.cpp:53, 67, 86-87, 129-166), written
// against include/qm_depthmap.hpp with QM_WITH_OPENCV.  Every statement that
// touches the Depthmap is written as those files write it, so this file
// compiling means those files compile against the drop-in unchanged.
//
// quadmap::SE3<float> is the reference's own type when QM_TEST_REFERENCE_SE3
// is defined (its include/ tree on the include path), else the stand-in
// below with the same members the callers use.
// Exit codes: 0 ok, 3 no CUDA device (QM_ERR_CUDA at construction), 1 failure.
#include <cmath>
#include <cstdio>
#include <memory>
#include <mutex>

#include "qm_depthmap.hpp"

#ifdef QM_TEST_REFERENCE_SE3
#include <quadmap/se3.cuh>
#else
namespace quadmap
{
template <typename T>
struct Rows3x4
{
  T v[12];
  T &operator[](int i) { return v[i]; }
  T operator[](int i) const { return v[i]; }
};

// Rigid transform [R | t], row-major, as the reference's SE3 stores it.
template <typename T>
struct SE3
{
  Rows3x4<T> data;
  SE3() : data{{1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0}} {}
  // unit quaternion (w, x, y, z) and translation
  SE3(T w, T x, T y, T z, T tx, T ty, T tz)
  {
    const T r[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
                    2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                    2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)};
    const T t[3] = {tx, ty, tz};
    for (int row = 0; row < 3; ++row)
    {
      for (int c = 0; c < 3; ++c)
        data[4 * row + c] = r[3 * row + c];
      data[4 * row + 3] = t[row];
    }
  }
  SE3 inv() const
  {
    SE3 o;
    for (int row = 0; row < 3; ++row)
      for (int c = 0; c < 3; ++c)
        o.data[4 * row + c] = data[4 * c + row];
    for (int row = 0; row < 3; ++row)
      o.data[4 * row + 3] = -(o.data[4 * row] * data[3] + o.data[4 * row + 1] * data[7] +
                              o.data[4 * row + 2] * data[11]);
    return o;
  }
};
} // namespace quadmap
#endif

namespace
{

const int kW = 160, kH = 128;
const float kF = 98.0f;

// a fronto-parallel textured plane 3 m away, seen from x = tx
void render(cv::Mat &img, float tx)
{
  for (int y = 0; y < kH; ++y)
    for (int x = 0; x < kW; ++x)
    {
      const float X = (x - 80.0f) / kF * 3.0f + tx;
      const float Y = (y - 64.0f) / kF * 3.0f;
      img.at<uint8_t>(y, x) = (uint8_t)(127 + 60 * std::sin(7.1f * X) * std::cos(5.3f * Y) +
                                        50 * std::sin(23.0f * X + 11.0f * Y));
    }
}

} // namespace

int main()
{
  try
  {
    // DepthmapNode::init (depthmap_node.cpp:95)
    const int resize_width = kW, resize_height = kH, semi2dense_ratio = 1;
    const float resize_fx = kF, resize_cx = 80.0f, resize_fy = kF, resize_cy = 64.0f;
    cv::Mat undist_map1, undist_map2;
    std::shared_ptr<quadmap::Depthmap> depthmap_ = std::make_shared<quadmap::Depthmap>(
        resize_width, resize_height, resize_fx, resize_cx, resize_fy, resize_cy, undist_map1,
        undist_map2, semi2dense_ratio);

    int results = 0, points = 0;
    bool pose_ok = true, maps_ok = true;
    cv::Mat img_8uC1(kH, kW, CV_8UC1);
    for (int f = 0; f < 40; ++f)
    {
      const float tx = 0.05f * f;
      render(img_8uC1, tx);
      // DepthmapNode::Msg_Callback (depthmap_node.cpp:127-138)
      quadmap::SE3<float> T_world_curr(1.0f, 0.0f, 0.0f, 0.0f, tx, 0.0f, 0.0f);
      bool has_result;
      has_result = depthmap_->add_frames(img_8uC1, T_world_curr.inv());
      if (!has_result)
        continue;
      ++results;
      // Publisher::publishDepthmap (publisher.cpp:53, 67, 86-87)
      cv::Mat debug_mat = depthmap_->getDebugmap();
      cv::Mat depthmap_mat = depthmap_->getDepthmap();
      cv::Mat reference_mat = depthmap_->getReferenceImage();
      maps_ok = maps_ok && debug_mat.rows == kH && depthmap_mat.cols == kW &&
                reference_mat.at<uint8_t>(10, 10) == img_8uC1.at<uint8_t>(10, 10);
      // Publisher::publishPointCloud (publisher.cpp:129-166)
      {
        std::lock_guard<std::mutex> lock(depthmap_->getRefImgMutex());

        const cv::Mat depth = depthmap_->getDepthmap();
        const cv::Mat ref_img = depthmap_->getReferenceImage();
        const quadmap::SE3<float> T_world_ref = depthmap_->getT_world_ref();

        const float fx = depthmap_->getFx();
        const float fy = depthmap_->getFy();
        const float cx = depthmap_->getCx();
        const float cy = depthmap_->getCy();
        pose_ok = pose_ok && T_world_ref.data[3] == tx && T_world_ref.data[0] == 1.0f;
        points = 0;
        for (int y = 0; y < depth.rows; ++y)
          for (int x = 0; x < depth.cols; ++x)
          {
            const float depth_value = depth.at<float>(y, x);
            if (depth_value < 0.1)
              continue;
            // the ray's z component, as the publisher normalises it
            const float rx = (x - cx) / fx, ry = (y - cy) / fy;
            const float z = depth_value / std::sqrt(rx * rx + ry * ry + 1.0f);
            if (z > 2.0f && z < 4.0f && ref_img.at<uint8_t>(y, x) == img_8uC1.at<uint8_t>(y, x))
              ++points;
          }
      }
    }
    std::printf("results=%d points=%d pose_ok=%d maps_ok=%d size=%zux%zu\n", results, points,
                (int)pose_ok, (int)maps_ok, depthmap_->getWidth(), depthmap_->getHeight());
    return (results >= 20 && points > 0 && pose_ok && maps_ok) ? 0 : 1;
  }
  catch (const quadmap::QmError &e)
  {
    std::printf("%s\n", e.what());
    return e.status == QM_ERR_CUDA ? 3 : 1;
  }
}
