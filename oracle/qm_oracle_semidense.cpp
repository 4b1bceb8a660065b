// TEST INFRASTRUCTURE ONLY (part of the oracle, linked into
// libqm_oracle.so with qm_oracle.cpp): a CPU restatement of the reference's
// semi-dense tracker (lsd_semidense.cu, seed_init.cu, host sequence
// seed_matrix.cu:106-146,211-446) in float IEEE arithmetic (build with
// -ffp-contract=off).  Used by tests/ as the checker of the device kernels.
//
// Where the reference's kernels race (in-place regularisation and hole
// filling, atomicCAS propagation with five retries, last-writer-wins
// projection) this restatement is deterministic: neighbourhood passes read
// the state before the pass, a propagation collision keeps the largest
// inverse depth (ties: larger source index), a projection collision the
// smallest depth (ties: smaller source index).  Bilinear image samples follow
// the texture unit's 8-bit weight arithmetic (SdFrame::sample) with clamp
// addressing.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

extern "C" int orc_get_threads(void);

namespace
{

template <class Fn>
void sd_par_for(int n, Fn &&f)
{
  const int T = std::min(orc_get_threads(), n);
  if (T <= 1)
  {
    for (int i = 0; i < n; ++i)
      f(i);
    return;
  }
  std::atomic<int> next(0);
  std::vector<std::thread> pool;
  for (int t = 0; t < T; ++t)
    pool.emplace_back([&]() {
      int i;
      while ((i = next.fetch_add(1)) < n)
        f(i);
    });
  for (auto &th : pool)
    th.join();
}

// float -> int truncation with saturation, NaN -> 0 (cvt.rzi.s32.f32)
inline int f2i_rz(float v)
{
  if (std::isnan(v))
    return 0;
  if (v >= 2147483648.0f)
    return 2147483647;
  if (v <= -2147483648.0f)
    return (-2147483647 - 1);
  return (int)v;
}

// double -> int likewise (cvt.rzi.s32.f64)
inline int d2i_rz(double v)
{
  if (std::isnan(v))
    return 0;
  if (v >= 2147483647.0)
    return 2147483647;
  if (v <= -2147483648.0)
    return (-2147483647 - 1);
  return (int)v;
}

struct SdSeed
{
  float t[4]; // valid (> 0), blacklist, validity counter, -
  float d[4]; // idepth, variance, smooth idepth, smooth variance
};

inline SdSeed sd_zero()
{
  SdSeed s;
  std::memset(&s, 0, sizeof(s));
  return s;
}

// DepthSeed::initialize (DepthSeed.cuh:15-26)
inline SdSeed sd_init(float idepth, float var, float counter)
{
  SdSeed s = sd_zero();
  s.t[0] = 1.0f;
  s.t[2] = counter;
  s.d[0] = idepth;
  s.d[1] = var;
  s.d[2] = 1.0f;
  s.d[3] = 4.0f;
  return s;
}

inline bool sd_valid(const SdSeed &s) { return s.t[0] > 0.0f; }

struct SdFrame
{
  int W, H;
  float fx, fy, cx, cy;
  std::vector<float> key, inc; // float images
  const float *T;              // T_income<-key
  float tex(const std::vector<float> &img, int x, int y) const { return img[(size_t)y * W + x]; }
  // tex2D with linear filtering, unnormalised coordinates, clamp addressing,
  // in the texture unit's arithmetic as measured on a B200: 256 a and 256 b
  // rounded half up to integers, the corner weights (1-a)(1-b) and ab
  // rounded half up to 1/256, a(1-b) and (1-a)b half down (they sum to
  // one), the weighted sum of the texels exact.
  static float round_frac8(float t)
  {
    const float f = std::floor(t);
    return (t - f) >= 0.5f ? f + 1.0f : f;
  }
  float sample(const std::vector<float> &img, float u, float v) const
  {
    const float xb = u - 0.5f, yb = v - 0.5f;
    const float fx0 = std::floor(xb), fy0 = std::floor(yb);
    const float A = round_frac8((xb - fx0) * 256.0f), B = round_frac8((yb - fy0) * 256.0f);
    const float nA = 256.0f - A, nB = 256.0f - B;
    const float w00 = std::floor(nA * nB * (1.0f / 256.0f) + 0.5f);
    const float w10 = std::ceil(A * nB * (1.0f / 256.0f) - 0.5f);
    const float w01 = std::ceil(nA * B * (1.0f / 256.0f) - 0.5f);
    const float w11 = std::floor(A * B * (1.0f / 256.0f) + 0.5f);
    const int i0 = f2i_rz(fx0), j0 = f2i_rz(fy0);
    const int xa = std::min(std::max(i0, 0), W - 1);
    const int xc = std::min(std::max(i0 == 2147483647 ? i0 : i0 + 1, 0), W - 1);
    const int ya = std::min(std::max(j0, 0), H - 1);
    const int yc = std::min(std::max(j0 == 2147483647 ? j0 : j0 + 1, 0), H - 1);
    float r = w00 * tex(img, xa, ya);
    r = r + w10 * tex(img, xc, ya);
    r = r + w01 * tex(img, xa, yc);
    r = r + w11 * tex(img, xc, yc);
    return r * (1.0f / 256.0f);
  }
  // gradient_kernel (seed_init.cu:26-41)
  void grad(const std::vector<float> &img, int x, int y, float &gx, float &gy) const
  {
    gx = (float)((double)(tex(img, x + 1, y) - tex(img, x - 1, y)) / 2.0);
    gy = (float)((double)(tex(img, x, y + 1) - tex(img, x, y - 1)) / 2.0);
  }
  // the seed kernels' range 2 < x < W-3, 2 < y < H-3
  bool interior(int x, int y) const { return !(x >= W - 3 || y >= H - 3 || x <= 2 || y <= 2); }
};

// search_point (lsd_semidense.cu:517-754)
float sd_search(const SdFrame &F, int x, int y, float ex, float ey, float gradient_max,
                float my_gradient, float min_idep, float max_idep, float &result_idep,
                float &result_var)
{
  const float fx = F.fx, fy = F.fy, cx = F.cx, cy = F.cy;
  const float *T = F.T;
  float this_patch[5];
  for (int i = -2; i <= 2; i++)
  {
    const float px = (float)x + (float)i * ex, py = (float)y + (float)i * ey;
    this_patch[i + 2] = F.sample(F.key, (float)((double)px + 0.5), (float)((double)py + 0.5));
  }
  // far and near points of the search range (:562-571)
  const float kx = ((float)x - cx) / fx, ky = ((float)y - cy) / fy, kz = 1.0f;
  const float rx = T[0] * kx + T[1] * ky + T[2] * kz;
  const float ry = T[4] * kx + T[5] * ky + T[6] * kz;
  const float rz = T[8] * kx + T[9] * ky + T[10] * kz;
  const float tx = T[3], ty = T[7], tz = T[11];
  const float Px = fx * rx + cx * rz, Py = fy * ry + cy * rz, Pz = rz;
  const float Kx = fx * tx + cx * tz, Ky = fy * ty + cy * tz, Kz = tz;
  const float nearx = Px + Kx * max_idep, neary = Py + Ky * max_idep, nearz = Pz + Kz * max_idep;
  const float farx = Px + Kx * min_idep, fary = Py + Ky * min_idep, farz = Pz + Kz * min_idep;
  float near_u = nearx / nearz, near_v = neary / nearz;
  float far_u = farx / farz, far_v = fary / farz;
  const float du = near_u - far_u, dv = near_v - far_v;
  float search_length = std::sqrt(du * du + dv * dv);
  const float dir_u = du / search_length, dir_v = dv / search_length;
  if ((double)search_length < 3.0)
  {
    near_u = near_u + dir_u * 2.0f;
    near_v = near_v + dir_v * 2.0f;
    far_u = far_u - dir_u * 2.0f;
    far_v = far_v - dir_v * 2.0f;
    search_length = (float)((double)search_length + 4.0);
  }
  if (far_u <= 1.0f || far_v <= 1.0f || far_u >= (float)(F.W - 2) || far_v >= (float)(F.H - 2))
    return -1.0f;
  float that_patch[5];
  for (int i = -2; i <= 1; i++)
  {
    const float px = far_u + (float)i * dir_u, py = far_v + (float)i * dir_v;
    that_patch[i + 2] = F.sample(F.inc, (float)((double)px + 0.5), (float)((double)py + 0.5));
  }
  // the search (:594-680)
  float best_step = -1.0f, best_score = 1e9f, pre_best_score = 1e9f, post_best_score = 1e9f;
  bool last_is_best = false;
  float best_pre = NAN, best_post = NAN;
  float e1A = NAN, e1B = NAN, e2A = NAN, e2B = NAN, e3A = NAN, e3B = NAN, e4A = NAN, e4B = NAN,
        e5A = NAN, e5B = NAN;
  float second_best_score = 1e9f, second_best_step = -1.0f;
  float pre_score = 1e9f, this_score = 1e9f;
  for (int step = 0; (float)step <= search_length && step <= 100; step += 1)
  {
    pre_score = this_score;
    this_score = 0.0f;
    const float sx = far_u + (float)step * dir_u, sy = far_v + (float)step * dir_v;
    if (sx <= 1.0f || sx >= (float)(F.W - 1) || sy <= 1.0f || sy >= (float)(F.H - 1))
      break;
    that_patch[4] = F.sample(F.inc, (float)((double)sx + 2.0 * (double)dir_u + 0.5),
                             (float)((double)sy + 2.0 * (double)dir_v + 0.5));
    if (step % 2 == 0)
    {
      e1A = that_patch[4] - this_patch[4];
      this_score = this_score + e1A * e1A;
      e2A = that_patch[3] - this_patch[3];
      this_score = this_score + e2A * e2A;
      e3A = that_patch[2] - this_patch[2];
      this_score = this_score + e3A * e3A;
      e4A = that_patch[1] - this_patch[1];
      this_score = this_score + e4A * e4A;
      e5A = that_patch[0] - this_patch[0];
      this_score = this_score + e5A * e5A;
    }
    else
    {
      e1B = that_patch[4] - this_patch[4];
      this_score = this_score + e1B * e1B;
      e2B = that_patch[3] - this_patch[3];
      this_score = this_score + e2B * e2B;
      e3B = that_patch[2] - this_patch[2];
      this_score = this_score + e3B * e3B;
      e4B = that_patch[1] - this_patch[1];
      this_score = this_score + e4B * e4B;
      e5B = that_patch[0] - this_patch[0];
      this_score = this_score + e5B * e5B;
    }
    if (last_is_best)
    {
      post_best_score = this_score;
      best_post = e1A * e1B + e2A * e2B + e3A * e3B + e4A * e4B + e5A * e5B;
      last_is_best = false;
    }
    if (this_score < best_score)
    {
      second_best_score = best_score;
      second_best_step = best_step;
      best_score = this_score;
      best_step = (float)step;
      pre_best_score = pre_score;
      best_pre = e1A * e1B + e2A * e2B + e3A * e3B + e4A * e4B + e5A * e5B;
      best_post = -1.0f;
      post_best_score = 1e9f;
      last_is_best = true;
    }
    else if (this_score < second_best_score)
    {
      second_best_score = this_score;
      second_best_step = (float)step;
    }
    that_patch[0] = that_patch[1];
    that_patch[1] = that_patch[2];
    that_patch[2] = that_patch[3];
    that_patch[3] = that_patch[4];
  }
  if (best_score > 4.0f * 1300.0f)
    return -3.0f;
  if (std::fabs(second_best_step - best_step) > 1.0f && 1.5f * best_score > second_best_score)
    return -2.0f;
  // sub-pixel refinement (:693-732)
  float best_match_sub = best_step;
  bool did_subpixel = false;
  {
    const float gpp = -(pre_best_score - best_pre);
    const float gpt = best_score - best_pre;
    const float gqt = -(best_score - best_post);
    const float gqq = post_best_score - best_post;
    bool interp_post = false, interp_pre = false;
    if ((gpp < 0.0f) ^ (gpt < 0.0f))
    {
      if (!((gqq < 0.0f) ^ (gqt < 0.0f)))
        interp_pre = true;
    }
    else if ((gqq < 0.0f) ^ (gqt < 0.0f))
      interp_post = true;
    if (interp_pre)
    {
      const float d = gpt / (gpt - gpp);
      best_match_sub = best_match_sub - d;
      best_score = best_score - 2.0f * d * gpt - (gpp - gpt) * d * d;
      did_subpixel = true;
    }
    else if (interp_post)
    {
      const float d = gqt / (gqt - gqq);
      best_match_sub = best_match_sub - d;
      best_score = best_score + 2.0f * d * gqt + (gqq - gqt) * d * d;
      did_subpixel = true;
    }
  }
  float gal = 0.0f;
  for (int i = 1; i < 5; i++)
    gal = gal + (this_patch[i] - this_patch[i - 1]) * (this_patch[i] - this_patch[i - 1]);
  if (best_score > 1300.0f + std::sqrt(gal) * 20.0f)
    return -3.0f;
  // inverse depth of the match and its variance (:734-752)
  float best_idepth, alpha;
  if (dir_u * dir_u > dir_v * dir_v)
  {
    const float bu = far_u + best_match_sub * dir_u;
    best_idepth = (bu * Pz - Px) / (Kx - bu * Kz);
    alpha = (Pz * Kx - Kz * Px) / ((Kx - bu * Kz) * (Kx - bu * Kz));
  }
  else
  {
    const float bv = far_v + best_match_sub * dir_v;
    best_idepth = (bv * Pz - Py) / (Ky - bv * Kz);
    alpha = (Pz * Ky - Kz * Py) / ((Ky - bv * Kz) * (Ky - bv * Kz));
  }
  best_idepth = (double)best_idepth < 0.01 ? 0.01f : best_idepth;
  best_idepth = (double)best_idepth > 2.0 ? 2.0f : best_idepth;
  const float photo = 16.0f / my_gradient / my_gradient;
  const float geo = 0.25f * gradient_max * gradient_max / (my_gradient * my_gradient);
  const double sub = did_subpixel ? 0.05 : 0.5;
  result_var = (float)((double)(alpha * alpha) * (sub + (double)geo + (double)photo));
  result_idep = best_idepth;
  return best_score;
}

// update_keyframe_kernel (lsd_semidense.cu:400-515), in place
void sd_update(const SdFrame &F, std::vector<SdSeed> &S)
{
  const float *T = F.T;
  sd_par_for(F.H, [&](int y) {
    for (int x = 0; x < F.W; ++x)
    {
      if (!F.interior(x, y))
        continue;
      float gx, gy;
      F.grad(F.key, x, y, gx, gy);
      const float gradient_max = std::sqrt(gx * gx + gy * gy);
      if (gradient_max < 5.0f)
        continue;
      SdSeed s = S[(size_t)y * F.W + x];
      if (s.t[1] < -1.0f)
        continue;
      const bool first_observe = !sd_valid(s);
      // translation of the inverse of T (se3.cuh:91-107)
      const float itx = -T[0] * T[3] - T[4] * T[7] - T[8] * T[11];
      const float ity = -T[1] * T[3] - T[5] * T[7] - T[9] * T[11];
      const float itz = -T[2] * T[3] - T[6] * T[7] - T[10] * T[11];
      float ex = -F.fx * itx + itz * ((float)x - F.cx);
      float ey = -F.fy * ity + itz * ((float)y - F.cy);
      const float epi_length = std::sqrt(ex * ex + ey * ey);
      if ((double)epi_length < 1.0)
        continue;
      ex = ex / epi_length;
      ey = ey / epi_length;
      const float gae = std::fabs(ex * gx + ey * gy);
      if ((double)gae < 2.0)
        continue;
      if ((double)(gae / gradient_max) < 0.3)
        continue;
      // the narrowed range of :451-458 lives in an inner scope: the search
      // always spans [MIN_INV_DEPTH, MAX_INV_DEPTH]
      float result_idep = 0.0f, result_var = 0.0f;
      const float err =
          sd_search(F, x, y, ex, ey, gradient_max, gae, 0.01f, 2.0f, result_idep, result_var);
      const float diff = result_idep - s.d[2];
      if (first_observe)
      {
        if (err == -3.0f || err == -2.0f)
          s.t[1] = s.t[1] - 1.0f;
        if (err > 0.0f && (double)result_var < 4.0)
          s = sd_init(result_idep, result_var, 5.0f);
      }
      else
      {
        if (err == -2.0f)
        {
          s.t[2] = s.t[2] - 5.0f;
          s.t[2] = s.t[2] < 0.0f ? 0.0f : s.t[2];
          s.d[1] = s.d[1] * 1.1f;
          if ((double)s.d[1] > 4.0)
          {
            s.t[0] = -1.0f;
            s.t[1] = s.t[1] - 1.0f;
          }
        }
        else if (err == -1.0f || err == -3.0f || err == -4.0f)
          continue;
        else if (diff * diff > result_var + s.d[3])
        {
          s.d[1] = s.d[1] * 1.1f;
          if ((double)s.d[1] > 4.0)
            s.t[0] = -1.0f;
        }
        else
        {
          const float inc_var = s.d[1] * 1.01f;
          const float new_var = (inc_var * result_var) / (inc_var + result_var);
          const float new_idepth =
              (s.d[0] * result_var + result_idep * inc_var) / (inc_var + result_var);
          if (new_var < s.d[1])
            s.d[1] = new_var;
          s.d[0] = new_idepth;
          s.t[2] = s.t[2] + 5.0f;
          const float max_valid = 5.0f + gradient_max * 250.0f / 255.0f;
          s.t[2] = s.t[2] > max_valid ? max_valid : s.t[2];
        }
      }
      S[(size_t)y * F.W + x] = s;
    }
  });
}

// regulizeDepth_FillHoles_kernel (lsd_semidense.cu:342-383), src -> dst; the
// gradient test reads the incoming image (:349)
void sd_fill(const SdFrame &F, const std::vector<SdSeed> &src, std::vector<SdSeed> &dst)
{
  sd_par_for(F.H, [&](int y) {
    for (int x = 0; x < F.W; ++x)
    {
      const size_t o = (size_t)y * F.W + x;
      SdSeed s = src[o];
      if (F.interior(x, y) && !sd_valid(s))
      {
        float gx, gy;
        F.grad(F.inc, x, y, gx, gy);
        if (!(gx * gx + gy * gy < 25.0f))
        {
          float sum_idepth = 0.0f, sum_ivar = 0.0f, sum_valid = 0.0f;
          for (int j = -2; j <= 2; j++)
            for (int i = -2; i <= 2; i++)
            {
              const SdSeed &n = src[o + (long)j * F.W + i];
              if (sd_valid(n))
              {
                sum_valid = sum_valid + n.t[2];
                const float w = 1.0f / n.d[1];
                sum_idepth = sum_idepth + n.d[0] * w;
                sum_ivar = sum_ivar + w;
              }
            }
          if (sum_valid > 100.0f || (s.t[1] >= -1.0f && sum_valid > 24.0f))
            s = sd_init(sum_idepth / sum_ivar, 1.0f / sum_ivar, 0.0f);
        }
      }
      dst[o] = s;
    }
  });
}

// regulizeDepth_kernel (lsd_semidense.cu:284-341), src -> dst
void sd_regularize(const SdFrame &F, const std::vector<SdSeed> &src, std::vector<SdSeed> &dst,
                   bool remove_occlusions)
{
  const float reg = 0.075f * 0.075f;
  sd_par_for(F.H, [&](int y) {
    for (int x = 0; x < F.W; ++x)
    {
      const size_t o = (size_t)y * F.W + x;
      SdSeed s = src[o];
      if (F.interior(x, y) && sd_valid(s))
      {
        float sum_idepth = 0.0f, sum_ivar = 0.0f, sum_valid = 0.0f;
        int occlusion = 0, not_occlusion = 0;
        for (int j = -2; j <= 2; j++)
          for (int i = -2; i <= 2; i++)
          {
            const SdSeed &n = src[o + (long)j * F.W + i];
            if (!sd_valid(n))
              continue;
            const float diff = s.d[0] - n.d[0];
            if (diff * diff > s.d[1] + n.d[1])
            {
              if (s.d[0] < n.d[0])
                occlusion++;
              continue;
            }
            sum_valid = sum_valid + n.t[2];
            not_occlusion++;
            const float spatial = reg * (float)(i * i + j * j);
            const float ivar = 1.0f / (n.d[1] + spatial);
            sum_idepth = sum_idepth + ivar * n.d[0];
            sum_ivar = sum_ivar + ivar;
          }
        if (sum_valid < 24.0f)
          s.t[0] = -1.0f;
        if (remove_occlusions && occlusion > not_occlusion)
          s.t[0] = -1.0f;
        s.d[2] = sum_idepth / sum_ivar;
        s.d[3] = 1.0f / sum_ivar;
      }
      dst[o] = s;
    }
  });
}

// the projection and gates shared by depth_project_kernel (:180-235) and
// propogate_keyframe_kernel (:100-146)
bool sd_project_seed(const SdFrame &F, int x, int y, float sidepth, float &px, float &py,
                     float &pz, float &new_idepth, int &nx, int &ny)
{
  float kx = ((float)x - F.cx) / F.fx, ky = ((float)y - F.cy) / F.fy, kz = 1.0f;
  kx = kx / sidepth;
  ky = ky / sidepth;
  kz = kz / sidepth;
  const float *T = F.T;
  px = T[0] * kx + T[1] * ky + T[2] * kz + T[3];
  py = T[4] * kx + T[5] * ky + T[6] * kz + T[7];
  pz = T[8] * kx + T[9] * ky + T[10] * kz + T[11];
  new_idepth = 1.0f / pz;
  nx = d2i_rz((double)(px * new_idepth * F.fx + F.cx) + 0.5);
  ny = d2i_rz((double)(py * new_idepth * F.fy + F.cy) + 0.5);
  if (nx <= 2 || nx >= F.W - 3 || ny <= 2 || ny >= F.H - 3)
    return false;
  float gx, gy;
  F.grad(F.inc, nx, ny, gx, gy);
  const float g2 = gx * gx + gy * gy;
  if (g2 < 25.0f)
    return false;
  const float diff = F.tex(F.key, x, y) - F.tex(F.inc, nx, ny);
  return !(diff * diff > (40.0f * 40.0f + 0.5f * 0.5f * g2));
}

// depth_project_kernel (:180-235) into `debug` (zero elsewhere)
void sd_project(const SdFrame &F, const std::vector<SdSeed> &S, float *debug)
{
  const size_t P = (size_t)F.W * F.H;
  std::vector<uint64_t> key(P, ~0ull);
  for (int y = 0; y < F.H; ++y)
    for (int x = 0; x < F.W; ++x)
    {
      if (!F.interior(x, y))
        continue;
      const size_t o = (size_t)y * F.W + x;
      const SdSeed &s = S[o];
      if (!sd_valid(s) || s.t[2] < 20.0f)
        continue;
      float px, py, pz, nid;
      int nx, ny;
      if (!sd_project_seed(F, x, y, s.d[2], px, py, pz, nid, nx, ny))
        continue;
      const float depth = std::sqrt(px * px + py * py + pz * pz);
      if (depth != depth || (double)s.d[3] > 0.02)
        continue;
      uint32_t bits;
      std::memcpy(&bits, &depth, 4);
      const uint64_t k = ((uint64_t)bits << 32) | (uint32_t)o;
      uint64_t &slot = key[(size_t)ny * F.W + nx];
      slot = std::min(slot, k);
    }
  for (size_t o = 0; o < P; ++o)
  {
    if (key[o] == ~0ull)
      debug[o] = 0.0f;
    else
    {
      const uint32_t bits = (uint32_t)(key[o] >> 32);
      std::memcpy(&debug[o], &bits, 4);
    }
  }
}

inline uint32_t sd_ordered(float f)
{
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// propogate_keyframe_kernel + initialize_keyframe_kernel (:80-178): the new
// keyframe's seeds
void sd_propagate(const SdFrame &F, const std::vector<SdSeed> &S, std::vector<SdSeed> &out)
{
  const size_t P = (size_t)F.W * F.H;
  std::vector<uint64_t> key(P, ~0ull);
  for (int y = 0; y < F.H; ++y)
    for (int x = 0; x < F.W; ++x)
    {
      if (!F.interior(x, y))
        continue;
      const size_t o = (size_t)y * F.W + x;
      if (!sd_valid(S[o]))
        continue;
      float px, py, pz, nid;
      int nx, ny;
      if (!sd_project_seed(F, x, y, S[o].d[2], px, py, pz, nid, nx, ny))
        continue;
      const uint64_t k = ~(((uint64_t)sd_ordered(nid) << 32) | (uint32_t)o);
      uint64_t &slot = key[(size_t)ny * F.W + nx];
      slot = std::min(slot, k);
    }
  for (int y = 0; y < F.H; ++y)
    for (int x = 0; x < F.W; ++x)
    {
      const size_t o = (size_t)y * F.W + x;
      out[o] = sd_zero();
      if (key[o] == ~0ull || !F.interior(x, y))
        continue;
      const uint32_t src = (uint32_t)(~key[o] & 0xffffffffull);
      const int sx = (int)(src % (uint32_t)F.W), sy = (int)(src / (uint32_t)F.W);
      const SdSeed &s = S[src];
      float px, py, pz, nid;
      int nx, ny;
      sd_project_seed(F, sx, sy, s.d[2], px, py, pz, nid, nx, ny);
      float r = nid / s.d[2];
      r = r * r;
      r = r * r;
      out[o] = sd_init(nid, r * s.d[3], s.t[2]);
    }
}

} // namespace

extern "C" {

// Bilinear samples of a u8 image at n unnormalised coordinates (x, y pairs),
// the texture unit's formula with 8-bit fractional weights (test hook).
void orc_sd_sample(const uint8_t *img, int W, int H, const float *uv, int n, float *out)
{
  SdFrame F;
  F.W = W;
  F.H = H;
  F.inc.resize((size_t)W * H);
  for (size_t o = 0; o < F.inc.size(); ++o)
    F.inc[o] = (float)img[o];
  for (int k = 0; k < n; ++k)
    out[k] = F.sample(F.inc, uv[2 * k], uv[2 * k + 1]);
}

// One semi-dense step of one stream (seed_matrix.cu:106-146).  mode 1: the
// first frame (seeds from `inc`; `key` unused); 2: update (update_keyframe,
// seed_matrix.cu:401-446); 3: update, then propagation into `inc` as the new
// keyframe (create_new_keyframe, seed_matrix.cu:246-304).  trk / dep: W*H*4
// floats each, in and out.  debug: W*H projected depths (0 elsewhere).
// T: 12 floats T_income<-key.
void orc_sd_step(int W, int H, float fx, float fy, float cx, float cy, const uint8_t *key,
                 const uint8_t *inc, const float *T, int mode, float *trk, float *dep,
                 float *debug)
{
  SdFrame F;
  F.W = W;
  F.H = H;
  F.fx = fx;
  F.fy = fy;
  F.cx = cx;
  F.cy = cy;
  F.T = T;
  const size_t P = (size_t)W * H;
  F.inc.resize(P);
  F.key.resize(P);
  for (size_t o = 0; o < P; ++o)
  {
    F.inc[o] = (float)inc[o];
    F.key[o] = key ? (float)key[o] : 0.0f;
  }
  std::vector<SdSeed> S(P), U(P);
  for (size_t o = 0; o < P; ++o)
  {
    std::memcpy(S[o].t, trk + 4 * o, 16);
    std::memcpy(S[o].d, dep + 4 * o, 16);
  }
  if (mode == 1)
  {
    // initialize_keyframe_kernel (lsd_semidense.cu:61-78)
    for (int y = 0; y < H; ++y)
      for (int x = 0; x < W; ++x)
      {
        SdSeed s = sd_zero();
        if (F.interior(x, y))
        {
          float gx, gy;
          F.grad(F.inc, x, y, gx, gy);
          if (!(gx * gx + gy * gy < 25.0f))
            s = sd_init(1.0f, 4.0f, 20.0f);
        }
        S[(size_t)y * W + x] = s;
      }
    std::fill(debug, debug + P, 0.0f);
  }
  else
  {
    sd_update(F, S);
    sd_fill(F, S, U);
    sd_regularize(F, U, S, false);
    sd_project(F, S, debug);
    if (mode == 3)
    {
      sd_propagate(F, S, U);
      sd_regularize(F, U, S, true);
      sd_fill(F, S, U);
      sd_regularize(F, U, S, false);
    }
  }
  for (size_t o = 0; o < P; ++o)
  {
    std::memcpy(trk + 4 * o, S[o].t, 16);
    std::memcpy(dep + 4 * o, S[o].d, 16);
  }
}

} // extern "C"
