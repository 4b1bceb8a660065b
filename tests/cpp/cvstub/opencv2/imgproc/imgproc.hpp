// Minimal stand-in for the parts of OpenCV's cv::Mat that the Depthmap
// drop-in header (QM_WITH_OPENCV) and the reference's ROS callers use, so
// that those code paths compile and run in tests without OpenCV.  Not
// OpenCV: 2-D, single channel, row-contiguous, shared ownership of the
// pixels; cv::remap copies its source (the tests pass no distortion maps).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <vector>

#define CV_8UC1 0
#define CV_32FC1 5

namespace cv
{

typedef unsigned char uchar;

enum
{
  INTER_LINEAR = 1
};
enum
{
  BORDER_CONSTANT = 0
};

class Mat
{
public:
  int rows = 0, cols = 0;
  uchar *data = nullptr;
  size_t step = 0;

  Mat() = default;
  Mat(int r, int c, int type) { create(r, c, type); }

  void create(int r, int c, int type)
  {
    const size_t elem = type == CV_32FC1 ? 4 : 1;
    if (buf_ && rows == r && cols == c && elem_ == elem)
      return;
    rows = r;
    cols = c;
    elem_ = elem;
    step = (size_t)c * elem;
    buf_ = std::make_shared<std::vector<uchar>>(step * (size_t)r);
    data = buf_->data();
  }
  bool empty() const { return data == nullptr || rows == 0 || cols == 0; }
  size_t elemSize() const { return elem_; }
  int type() const { return elem_ == 4 ? CV_32FC1 : CV_8UC1; }

  template <class T>
  T &at(int y, int x)
  {
    return reinterpret_cast<T *>(data + (size_t)y * step)[x];
  }
  template <class T>
  const T &at(int y, int x) const
  {
    return reinterpret_cast<const T *>(data + (size_t)y * step)[x];
  }

  Mat clone() const
  {
    Mat m(rows, cols, type());
    if (!empty())
      std::memcpy(m.data, data, step * (size_t)rows);
    return m;
  }

private:
  std::shared_ptr<std::vector<uchar>> buf_;
  size_t elem_ = 1;
};

template <class T>
class Mat_ : public Mat
{
public:
  Mat_() = default;
  Mat_(int r, int c) { create(r, c); }
  Mat_(const Mat &m) : Mat(m) {}
  void create(int r, int c) { Mat::create(r, c, sizeof(T) == 4 ? CV_32FC1 : CV_8UC1); }
};

inline void remap(const Mat &src, Mat &dst, const Mat &map1, const Mat &, int, int)
{
  if (!map1.empty())
    throw std::runtime_error("cv stub: remap with distortion maps is not implemented");
  dst = src.clone();
}

} // namespace cv
