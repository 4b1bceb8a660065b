// TEST INFRASTRUCTURE ONLY: the point-cloud loop of the reference's
// Publisher::publishPointCloud (publisher.cpp:146-163) evaluated with the
// reference's own host arithmetic: normalize() and float3 operators of its
// cuda_toolkit/helper_math.h (host rsqrtf = 1 / sqrtf, helper_math.h:62-65)
// and SE3<float>::operator* of its quadmap/se3.cuh (se3.cuh:122-151,198-201),
// compiled with g++ from the reference headers where they lie (`make -C
// oracle ref-host`).  publisher.cpp itself needs ROS, PCL and OpenCV, so the
// loop around those calls is restated here.  Used only to make the golden
// point-cloud fixture (tests/golden/make_pointcloud_golden.py).
#include <cstdint>

#include <cuda_runtime.h>
#include <quadmap/se3.cuh>

extern "C" int qmref_point_cloud(const float *depth, const uint8_t *ref, int W, int H, float fx,
                                 float fy, float cx, float cy, const float *T, float *xyzi)
{
  quadmap::SE3<float> T_world_ref;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 4; ++c)
      T_world_ref.data(r, c) = T[4 * r + c];
  int n = 0;
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x)
    {
      const float depth_value = depth[(size_t)y * W + x];
      if (depth_value < 0.1)
        continue;
      const float3 f = normalize(make_float3((x - cx) / fx, (y - cy) / fy, 1.0f));
      const float3 xyz = T_world_ref * (f * depth_value);
      float *o = xyzi + 4 * (size_t)n;
      o[0] = xyz.x;
      o[1] = xyz.y;
      o[2] = xyz.z;
      o[3] = ref[(size_t)y * W + x];
      ++n;
    }
  return n;
}
