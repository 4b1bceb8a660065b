// C++ use of the drop-in header: builds a Depthmap, feeds a synthetic
// translating texture, reads the maps back.  Exit codes: 0 ok, 3 no CUDA
// device (the library reported QM_ERR_CUDA at construction), 1 failure.
#include <cmath>
#include <cstdio>
#include <vector>

#include "qm_depthmap.hpp"

struct Pose
{
  float data[12];
};

int main()
{
  const int W = 160, H = 128;
  try
  {
    quadmap::Depthmap dm(W, H, 98.0f, 80.0f, 98.0f, 64.0f, 1);
    std::vector<uint8_t> img(W * H);
    std::vector<float> depth(W * H);
    int results = 0;
    for (int f = 0; f < 14; ++f)
    {
      // a fronto-parallel textured plane 3 m away, camera sliding along x
      const float tx = -0.06f * f;
      for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
        {
          const float X = (x - 80.0f) / 98.0f * 3.0f - tx;
          const float Y = (y - 64.0f) / 98.0f * 3.0f;
          img[y * W + x] = (uint8_t)(127 + 60 * std::sin(7.1f * X) * std::cos(5.3f * Y) +
                                     50 * std::sin(23.0f * X + 11.0f * Y));
        }
      Pose T = {{1, 0, 0, tx, 0, 1, 0, 0, 0, 0, 1, 0}};
      if (dm.add_frames(img.data(), W, T.data))
        ++results;
    }
    dm.getDepthmap(depth.data(), W);
    std::printf("results=%d depth(80,64)=%.3f\n", results, depth[64 * W + 80]);
    return results >= 3 ? 0 : 1;
  }
  catch (const quadmap::QmError &e)
  {
    std::printf("%s\n", e.what());
    return e.status == QM_ERR_CUDA ? 3 : 1;
  }
}
