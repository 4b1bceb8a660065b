// TEST INFRASTRUCTURE ONLY.  This file is the oracle: a CPU restatement of
// the reference's per-keyframe depth pipeline (open_quadtree_mapping), used by
// tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm
// as the checker.  Nothing in the product imports, links or executes it.
//
// Each function follows a reference kernel step for step, in the same
// arithmetic order, with IEEE single-precision operations (no FMA
// contraction: build with -ffp-contract=off) and libm's expf/sqrtf.  The
// reference GPU build uses -use_fast_math, so its divisions, rsqrtf and expf
// are approximations; this oracle does not emulate them.  Expected
// agreement with the reference kernels: level map bit-exact; cost volume and
// BP labels equal except where a rounded projection falls within a
// fast-math error of a .5 boundary; depths within a small relative tolerance.
// The product's IEEE arithmetic mode reproduces this oracle bit-exactly for
// levels, costs, messages and labels.
//
// Every routine is templated on the real type R: R=float is the reference
// order (the "fp32 oracle"), R=double the same algorithm in double (the
// "fp64 oracle") used to state the error of every output.
//
// Parity pins: tests/golden/ holds dumps of the reference's own kernels
// (built from the reference sources by oracle/Makefile into oracle/_ref/ and
// run on a B200 by tests/golden/make_golden.py); tests check this oracle
// against them.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

namespace
{

int g_threads = 1;

// Runs f(i) for i in [0, n) on g_threads host threads (dynamic schedule).
template <class F>
void par_for(int n, F &&f)
{
  const int T = std::min(g_threads, n);
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

// Conversion double -> int as the GPU's cvt.rzi.s32.f64 does it: truncate
// toward zero, saturate to the int range, NaN -> 0.
inline int trunc_sat(double v)
{
  if (std::isnan(v))
    return 0;
  if (v >= 2147483647.0)
    return 2147483647;
  if (v <= -2147483648.0)
    return (-2147483647 - 1);
  return (int)v;
}

struct Cam
{
  float fx, fy, cx, cy;
};

} // namespace

extern "C" {

// Parameters shared by the oracle stages (a subset of the product's
// qm_params; the Python wrapper fills both from one dictionary).
struct orc_params
{
  int num_hyp;          // D, hypotheses per cell (reference DEPTH_NUM 64)
  double min_inv_depth; // reference MIN_INV_DEPTH 0.01
  double inv_depth_step;// reference STEP_INV_DEPTH (2.0-0.01)/63.0
  float P1, P2;         // bpextract.cu:222-223 (0.003, 0.01)
  int bp_levels;        // bpextract.cu:41 (4)
  int bp_iters[8];      // fine -> coarse, bpextract.cu:45 ({4,10,10,10})
  int qt_max_level;     // quadtree.cu:40 (4)
  int qt_min_level;     // quadtree.cu:74 (2)
  float qt_threshold;   // quadtree.cu:59 (10.0)
  double up_sigma;      // stereo_parameter.cuh (upsample_sigma 400.0)
  double up_lambda;     // stereo_parameter.cuh (upsample_lambda 10.0)
};

} // extern "C"

namespace
{

// ---------------------------------------------------------------------------
// Quadtree levels: quadtree.cu:17-77.
//
// A block of side 2^i aligned to 2^i is "approved" when it lies wholly inside
// the image, all four of its 2^(i-1) children are approved, and every pixel
// differs from the block mean by at most the threshold.  A pixel's level is
// the largest i <= max_level whose containing block is approved, clamped to
// at least min_level.  (In the kernel, a pixel whose sub-block fails exits,
// which makes the pixel count of every enclosing block fall short; that is
// the "all children approved" condition.)  Sums of <= 4^max_level integer
// intensities are exact in float and the mean divides by a power of two, so
// the result does not depend on summation order.
void quadtree_levels(const uint8_t *img, int w, int h, int max_level, int min_level,
                     float thr, int *levels)
{
  std::vector<uint8_t> ok_prev, ok_cur;
  // Level 0: every pixel is its own approved block.
  int bw_prev = w, bh_prev = h;
  ok_prev.assign((size_t)w * h, 1);
  for (int p = 0; p < w * h; ++p)
    levels[p] = 0;
  for (int i = 1; i <= max_level; ++i)
  {
    const int s = 1 << i;
    const int bw = (w + s - 1) / s, bh = (h + s - 1) / s;
    ok_cur.assign((size_t)bw * bh, 0);
    const float inv_n = 1.0f / (float)(s * s);
    for (int by = 0; by < bh; ++by)
      for (int bx = 0; bx < bw; ++bx)
      {
        const int x0 = bx * s, y0 = by * s;
        if (x0 + s > w || y0 + s > h)
          continue; // incomplete block
        bool children = true;
        for (int cy = 0; cy < 2; ++cy)
          for (int cx = 0; cx < 2; ++cx)
          {
            int cbx = 2 * bx + cx, cby = 2 * by + cy;
            if (!ok_prev[(size_t)cby * bw_prev + cbx])
              children = false;
          }
        if (!children)
          continue;
        float sum = 0.0f;
        for (int y = y0; y < y0 + s; ++y)
          for (int x = x0; x < x0 + s; ++x)
            sum += (float)img[(size_t)y * w + x];
        const float mean = sum * inv_n;
        bool good = true;
        for (int y = y0; y < y0 + s && good; ++y)
          for (int x = x0; x < x0 + s; ++x)
            if ((double)std::fabs((float)img[(size_t)y * w + x] - mean) > (double)thr)
            {
              good = false;
              break;
            }
        if (!good)
          continue;
        ok_cur[(size_t)by * bw + bx] = 1;
        for (int y = y0; y < y0 + s; ++y)
          for (int x = x0; x < x0 + s; ++x)
            levels[(size_t)y * w + x] = i;
      }
    ok_prev.swap(ok_cur);
    bw_prev = bw;
    bh_prev = bh;
  }
  for (int p = 0; p < w * h; ++p)
    if (levels[p] < min_level)
      levels[p] = min_level;
}

// ---------------------------------------------------------------------------
// Matching cost: depth_extract.cu:135-244 (image_to_cost + normalize_the_cost).
//
// Cells are 4x4; cell (cx, cy) is evaluated at pixel (4cx, 4cy) when that
// pixel is a quadtree node origin and not on the image border
// (depth_extract.cu:150).  For hypothesis d the pixel's viewing ray
// (normalised K^-1 [x y 1]) is scaled to depth 1/(min + step*d) (computed in
// double, stored in float), moved into measurement slot f by T_f (rotate then
// translate), projected, rounded by truncating +0.5, and, when inside
// [2, W-2) x [2, H-2), scored by the SAD of the 3x3 reference patch against
// the 3x3 measurement patch whose offsets are rotated by the top-left 2x2 of
// R_f (depth_extract.cu:183-199).  The cost is sum/n_valid/255, or 100 when
// no slot is valid, then divided by the number of hypotheses (the writer
// count normalize_the_cost divides by).  Every term of the SAD is an integer,
// so the sum is exact in any order.
template <typename R>
void cost_volume(const uint8_t *ref, int w, int h, const int *levels, int nslots,
                 const uint8_t *const *slot_img, const float *T, const Cam &cam,
                 const orc_params &p, R *cost, int *valid_cells)
{
  const int cw = w / 4, ch = h / 4, D = p.num_hyp;
  par_for(ch, [&](int cy) {
    std::vector<R> hyp_depth(D);
    for (int d = 0; d < D; ++d)
    {
      double dd = 1.0 / (p.inv_depth_step * (double)d + p.min_inv_depth);
      hyp_depth[d] = (R)dd;
    }
    for (int cx = 0; cx < cw; ++cx)
    {
      const int x = cx * 4, y = cy * 4;
      R *out = cost + ((size_t)cy * cw + cx) * D;
      for (int d = 0; d < D; ++d)
        out[d] = 0;
      if (valid_cells)
        valid_cells[(size_t)cy * cw + cx] = 0;
      const int size = 1 << levels[(size_t)y * w + x];
      if (x >= w - 1 || y >= h - 1 || x <= 0 || y <= 0 || x % size != 0 || y % size != 0)
        continue;
      if (valid_cells)
        valid_cells[(size_t)cy * cw + cx] = 1;
      int patch[3][3];
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i)
          patch[i][j] = ref[(size_t)(y + j - 1) * w + (x + i - 1)];
      // normalize(cam2world(x, y)); host helper_math: v * (1/sqrt(dot(v,v)))
      const R vx = ((R)x - (R)cam.cx) / (R)cam.fx;
      const R vy = ((R)y - (R)cam.cy) / (R)cam.fy;
      const R vz = (R)1;
      const R dot = vx * vx + vy * vy + vz * vz;
      const R inv_len = (R)1 / std::sqrt(dot);
      const R dx = vx * inv_len, dy = vy * inv_len, dz = vz * inv_len;
      for (int d = 0; d < D; ++d)
      {
        const R depth = hyp_depth[d];
        const R px = dx * depth, py = dy * depth, pz = dz * depth;
        long sad = 0;
        int nvalid = 0;
        for (int f = 0; f < nslots; ++f)
        {
          const float *t = T + 12 * f;
          const R qx = (R)t[0] * px + (R)t[1] * py + (R)t[2] * pz + (R)t[3];
          const R qy = (R)t[4] * px + (R)t[5] * py + (R)t[6] * pz + (R)t[7];
          const R qz = (R)t[8] * px + (R)t[9] * py + (R)t[10] * pz + (R)t[11];
          const R u = (R)cam.fx * qx / qz + (R)cam.cx;
          const R v = (R)cam.fy * qy / qz + (R)cam.cy;
          const int pxi = trunc_sat((double)u + 0.5);
          const int pyi = trunc_sat((double)v + 0.5);
          if (!(pxi >= 2 && pxi < w - 2 && pyi >= 2 && pyi < h - 2))
            continue;
          const R u2u = (R)t[0], u2v = (R)t[4], v2u = (R)t[1], v2v = (R)t[5];
          const uint8_t *m = slot_img[f];
          int s = 0;
          for (int j = -1; j <= 1; ++j)
            for (int i = -1; i <= 1; ++i)
            {
              const int chx = trunc_sat((double)(u + u2u * (R)i + v2u * (R)j) + 0.5);
              const int chy = trunc_sat((double)(v + u2v * (R)i + v2v * (R)j) + 0.5);
              s += std::abs(patch[i + 1][j + 1] - (int)m[(size_t)chy * w + chx]);
            }
          sad += s;
          nvalid += 1;
        }
        R c;
        if (nvalid > 0)
          c = (R)sad / (R)nvalid / (R)255;
        else
          c = (R)100;
        // normalize_the_cost divides by the cell's writer count: every
        // hypothesis thread of slot row 0 adds 1 (depth_extract.cu:219-228),
        // so the count is the number of hypotheses.
        out[d] = c / (R)D;
      }
    }
  });
}

// ---------------------------------------------------------------------------
// Hierarchical belief propagation and extraction: bpextract.cu:37-395.

inline int pow2_ceil(int n)
{
  int p = 1;
  while (p < n)
    p <<= 1;
  return p;
}

// Stride-halving tree sum of bpextract.cu:293-300 (exact order), padded with
// zeros to the next power of two for hypothesis counts that are not one.
template <typename R>
R tree_sum(const R *v, int n, R *scratch)
{
  const int P = pow2_ceil(n);
  for (int i = 0; i < P; ++i)
    scratch[i] = i < n ? v[i] : (R)0;
  for (int s = P / 2; s > 0; s /= 2)
    for (int i = 0; i < s; ++i)
      scratch[i] += scratch[i + s];
  return scratch[0];
}

// Stride-halving tree argmin of bpextract.cu:347-355: at every node the right
// element wins only when strictly smaller.
template <typename R>
int tree_argmin(const R *v, int n, R *sv, int *si)
{
  const int P = pow2_ceil(n);
  for (int i = 0; i < P; ++i)
  {
    sv[i] = i < n ? v[i] : std::numeric_limits<R>::infinity();
    si[i] = i;
  }
  for (int s = P / 2; s > 0; s /= 2)
    for (int i = 0; i < s; ++i)
      if (sv[i + s] < sv[i])
      {
        sv[i] = sv[i + s];
        si[i] = si[i + s];
      }
  return si[0];
}

template <typename R>
struct Level
{
  int w, h;
  std::vector<R> data;          // [y][x][d]
  std::vector<R> up, down, left, right; // outgoing messages [y][x][d]
};

// One red-black half-sweep (bp kernel, bpextract.cu:200-312) over level lv.
template <typename R>
void bp_half_sweep(Level<R> &L, int D, bool a_set, int lv, const int *qt, int W, int H,
                   const orc_params &p)
{
  const int hw = (L.w + 1) / 2;
  const R P1 = (R)p.P1, P2 = (R)p.P2;
  const int i_lev = lv + 2;
  par_for(L.h, [&](int y) {
    std::vector<R> hcur(D), scratch(pow2_ceil(D) + 1), msg(D);
      for (int bx = 0; bx < hw; ++bx)
      {
        if (i_lev <= p.qt_max_level)
        {
          const int size = 1 << i_lev;
          const int sx = std::min(bx * size, W - 1), sy = std::min(y * size, H - 1);
          if (qt[(size_t)sy * W + sx] > i_lev)
            continue;
        }
        const int x = bx * 2 + (a_set ? (y % 2) : ((y + 1) % 2));
        if (x >= L.w || y >= L.h)
          continue;
        const size_t c = ((size_t)y * L.w + x) * D;
        const bool on_up = y == 0, on_down = y == L.h - 1, on_left = x == 0,
                   on_right = x == L.w - 1;
        for (int dir = 0; dir < 4; ++dir)
        {
          for (int d = 0; d < D; ++d)
          {
            R v = L.data[c + d];
            if (dir != 0 && !on_up)
              v += L.down[((size_t)(y - 1) * L.w + x) * D + d];
            if (dir != 1 && !on_down)
              v += L.up[((size_t)(y + 1) * L.w + x) * D + d];
            if (dir != 2 && !on_left)
              v += L.right[((size_t)y * L.w + (x - 1)) * D + d];
            if (dir != 3 && !on_right)
              v += L.left[((size_t)y * L.w + (x + 1)) * D + d];
            hcur[d] = v;
          }
          R hmin = hcur[0];
          for (int d = 1; d < D; ++d)
            hmin = hcur[d] < hmin ? hcur[d] : hmin;
          for (int d = 0; d < D; ++d)
          {
            R m = hcur[d];
            if (d > 0)
              m = std::min(m, hcur[d - 1] + P1);
            if (d < D - 1)
              m = std::min(m, hcur[d + 1] + P1);
            m = std::min(m, hmin + P2);
            msg[d] = m;
          }
          const R mean = tree_sum(msg.data(), D, scratch.data()) / (R)D;
          std::vector<R> &out = dir == 0 ? L.up : dir == 1 ? L.down : dir == 2 ? L.left : L.right;
          for (int d = 0; d < D; ++d)
            out[c + d] = msg[d] - mean;
        }
      }
  });
}

// bp_extract (bpextract.cu:37-167) followed by depth_extract
// (bpextract.cu:314-372).  labels[cell] = winning hypothesis at node-origin
// cells, -1 elsewhere; sparse (W x H) receives the depth at (4x, 4y) of every
// node-origin cell and is left untouched elsewhere.  msg_out (optional) gets
// the final level-0 messages in the order up, down, left, right.
template <typename R>
void bp_extract(const R *cost, int W, int H, const int *qt, const orc_params &p, int *labels,
                R *sparse, R *msg_out, double tau = 0.0)
{
  const int D = p.num_hyp, NL = p.bp_levels;
  std::vector<Level<R>> lv(NL);
  lv[0].w = W / 4;
  lv[0].h = H / 4;
  for (int i = 1; i < NL; ++i)
  {
    lv[i].w = (lv[i - 1].w + 1) / 2;
    lv[i].h = (lv[i - 1].h + 1) / 2;
  }
  lv[0].data.assign(cost, cost + (size_t)lv[0].w * lv[0].h * D);
  // cost_distribute (bpextract.cu:169-198): sum of the 2x2 children, x offset
  // outer, y offset inner, starting from zero.
  for (int i = 1; i < NL; ++i)
  {
    Level<R> &a = lv[i - 1], &b = lv[i];
    b.data.assign((size_t)b.w * b.h * D, (R)0);
    for (int y = 0; y < b.h; ++y)
      for (int x = 0; x < b.w; ++x)
        for (int d = 0; d < D; ++d)
        {
          R s = 0;
          for (int ii = 0; ii < 2; ++ii)
            for (int jj = 0; jj < 2; ++jj)
              if (2 * x + ii < a.w && 2 * y + jj < a.h)
                s += a.data[((size_t)(2 * y + jj) * a.w + (2 * x + ii)) * D + d];
          b.data[((size_t)y * b.w + x) * D + d] = s;
        }
  }
  for (int i = NL - 1; i >= 0; --i)
  {
    Level<R> &L = lv[i];
    const size_t n = (size_t)L.w * L.h * D;
    if (i == NL - 1)
    {
      L.up.assign(n, (R)0);
      L.down.assign(n, (R)0);
      L.left.assign(n, (R)0);
      L.right.assign(n, (R)0);
    }
    else
    {
      // upsample (bpextract.cu:374-395): every child copies its parent.
      Level<R> &C = lv[i + 1];
      L.up.resize(n);
      L.down.resize(n);
      L.left.resize(n);
      L.right.resize(n);
      for (int y = 0; y < L.h; ++y)
        for (int x = 0; x < L.w; ++x)
        {
          const size_t dst = ((size_t)y * L.w + x) * D;
          const size_t src = ((size_t)(y / 2) * C.w + (x / 2)) * D;
          for (int d = 0; d < D; ++d)
          {
            L.up[dst + d] = C.up[src + d];
            L.down[dst + d] = C.down[src + d];
            L.left[dst + d] = C.left[src + d];
            L.right[dst + d] = C.right[src + d];
          }
        }
      C.up.clear();
      C.down.clear();
      C.left.clear();
      C.right.clear();
    }
    bool a_set = true;
    for (int it = 0; it < p.bp_iters[i]; ++it)
    {
      bp_half_sweep(L, D, a_set, i, qt, W, H, p);
      a_set = !a_set;
    }
  }
  // depth_extract: belief = data + right-msg of the left neighbour + left-msg
  // of the right neighbour + down-msg of the upper + up-msg of the lower.
  Level<R> &L = lv[0];
  par_for(L.h, [&](int y) {
    std::vector<R> b(D), sv(pow2_ceil(D) + 1);
    std::vector<int> si(pow2_ceil(D) + 1);
      for (int x = 0; x < L.w; ++x)
      {
        const size_t cell = (size_t)y * L.w + x;
        labels[cell] = -1;
        const int lvl = qt[(size_t)std::min(y * 4, H - 1) * W + std::min(x * 4, W - 1)];
        const int size = 1 << lvl;
        if ((x * 4) % size != 0 || (y * 4) % size != 0)
          continue;
        for (int d = 0; d < D; ++d)
        {
          R v = L.data[cell * D + d];
          if (x != 0)
            v += L.right[(cell - 1) * D + d];
          if (x != L.w - 1)
            v += L.left[(cell + 1) * D + d];
          if (y != 0)
            v += L.down[(cell - L.w) * D + d];
          if (y != L.h - 1)
            v += L.up[(cell + L.w) * D + d];
          b[d] = v;
        }
        const int best = tree_argmin(b.data(), D, sv.data(), si.data());
        labels[cell] = best;
        R disparity = (R)best;
        if (best > 0 && best < D - 1)
        {
          const R pre = b[best - 1], post = b[best + 1];
          const R a = pre - (R)2 * b[best] + post;
          const R bb = -pre + post;
          const R b_a = bb / a;
          if (std::isfinite(b_a))
            disparity = (R)best - b_a / (R)2;
        }
        if (tau > 0.0)
        {
          // softened readout of the differentiable path (not in the
          // reference): disparity = sum_d softmax(-b/tau)(d) * d
          R bmin = b[0];
          for (int d = 1; d < D; ++d)
            bmin = std::min(bmin, b[d]);
          R z = 0, s = 0;
          for (int d = 0; d < D; ++d)
          {
            const R e = std::exp(-(b[d] - bmin) / (R)tau);
            z += e;
            s += e * (R)d;
          }
          disparity = s / z;
        }
        const double dep = 1.0 / (p.inv_depth_step * (double)disparity + p.min_inv_depth);
        sparse[(size_t)(y * 4) * W + x * 4] = (R)dep;
      }
  });
  if (msg_out)
  {
    const size_t n = (size_t)L.w * L.h * D;
    std::copy(L.up.begin(), L.up.end(), msg_out);
    std::copy(L.down.begin(), L.down.end(), msg_out + n);
    std::copy(L.left.begin(), L.left.end(), msg_out + 2 * n);
    std::copy(L.right.begin(), L.right.end(), msg_out + 3 * n);
  }
}

// ---------------------------------------------------------------------------
// Edge-aware upsampling: depth_upsample.cu:20-302 (global_upsample).

// build_weight_row / build_weight_col (depth_upsample.cu:58-93), including
// the launch-grid quirk: the grids cover ceil(W/16)*16 x ceil(H/16)*16
// threads, so row_w(W, .) (resp. col_w(., H)) is written as exp(0) = 1 when
// W (resp. H) is not a multiple of 16, and stays 0 otherwise.
template <typename R>
void upsample_weights(const uint8_t *img, int W, int H, const orc_params &p, R *row_w, R *col_w)
{
  const int gw = (W + 15) / 16 * 16, gh = (H + 15) / 16 * 16;
  auto I = [&](int x, int y) {
    x = std::min(std::max(x, 0), W - 1);
    y = std::min(std::max(y, 0), H - 1);
    return (R)img[(size_t)y * W + x];
  };
  std::fill(row_w, row_w + (size_t)(W + 1) * H, (R)0);
  std::fill(col_w, col_w + (size_t)W * (H + 1), (R)0);
  for (int y = 0; y < H; ++y)
    for (int x = 1; x < std::min(W + 1, gw); ++x)
    {
      const R diff = I(x, y) - I(x - 1, y);
      const R arg = (R)((double)(-diff * diff) / p.up_sigma);
      row_w[(size_t)y * (W + 1) + x] = std::exp(arg);
    }
  for (int y = 1; y < std::min(H + 1, gh); ++y)
    for (int x = 0; x < W; ++x)
    {
      const R diff = I(x, y) - I(x, y - 1);
      const R arg = (R)((double)(-diff * diff) / p.up_sigma);
      col_w[(size_t)y * W + x] = std::exp(arg);
    }
}

// Solve (I + lambda*L_w) s = r along one line of n samples for r = depth and
// r = indicator (depth > 0) with the Thomas algorithm in the order of
// smooth_row (depth_upsample.cu:94-197).  w[k] is the weight between samples
// k-1 and k (w[0] = 0); w[n] closes the line.
template <typename R>
void thomas_line(int n, const R *w, size_t wstride, const R *rd, const R *ri, size_t rstride,
                 R lambda, R *sd, R *si, bool indicator_from_depth)
{
  std::vector<R> ch(n), dh(n), ih(n);
  R fc = 0, fd = 0, fi = 0;
  for (int k = 0; k < n; ++k)
  {
    const R wl = k == 0 ? (R)0 : w[k * wstride];
    const R wr = w[(k + 1) * wstride];
    const R dep = rd[k * rstride];
    const R ind = indicator_from_depth ? (dep > 0 ? (R)1 : (R)0) : ri[k * rstride];
    const R a = (R)(-(double)lambda * (double)wl);
    const R b = (R)(1.0 + (double)lambda * (double)(wl + wr));
    const R c = (R)(-(double)lambda * (double)wr);
    const R den = b - fc * a;
    const R c_hat = c / den;
    const R d_hat = (dep - fd * a) / den;
    const R i_hat = (ind - fi * a) / den;
    fc = c_hat;
    fd = d_hat;
    fi = i_hat;
    ch[k] = c_hat;
    dh[k] = d_hat;
    ih[k] = i_hat;
  }
  R nd = 0, ni = 0;
  for (int k = n - 1; k >= 0; --k)
  {
    const R s_d = dh[k] - ch[k] * nd;
    const R s_i = ih[k] - ch[k] * ni;
    sd[k * rstride] = s_d;
    si[k * rstride] = s_i;
    nd = s_d;
    ni = s_i;
  }
}

// global_upsample: rows then columns, output S_col(S_row(d)) / S_col(S_row(1)).
// smooth_row only writes whole 16-sample chunks and smooth_col whole 8-row
// chunks; the tails (W % 16, H % 8) keep whatever the output held.
template <typename R>
void upsample(const R *sparse, const uint8_t *img, int W, int H, const orc_params &p, R *dense,
              const double *omega = nullptr)
{
  std::vector<R> row_w((size_t)(W + 1) * H), col_w((size_t)W * (H + 1));
  upsample_weights(img, W, H, p, row_w.data(), col_w.data());
  if (omega)
  {
    // per-pixel factors of the differentiable path (not in the reference):
    // the edge between a pixel and its left / upper neighbour is scaled by
    // the pixel's factor
    for (int y = 0; y < H; ++y)
      for (int x = 1; x < W; ++x)
        row_w[(size_t)y * (W + 1) + x] *= (R)omega[(size_t)y * W + x];
    for (int y = 1; y < H; ++y)
      for (int x = 0; x < W; ++x)
        col_w[(size_t)y * W + x] *= (R)omega[(size_t)y * W + x];
  }
  const int wr = W / 16 * 16, hr = H / 8 * 8;
  std::vector<R> rd((size_t)W * H, (R)0), ri((size_t)W * H, (R)0);
  const R lambda = (R)p.up_lambda;
  par_for(H, [&](int y) {
    if (wr == 0)
      return;
    // the row solve runs over the first wr samples, weight wr closes it
    std::vector<R> w(wr + 1);
    for (int k = 0; k <= wr; ++k)
      w[k] = row_w[(size_t)y * (W + 1) + k];
    thomas_line<R>(wr, w.data(), 1, sparse + (size_t)y * W, nullptr, 1, lambda,
                   rd.data() + (size_t)y * W, ri.data() + (size_t)y * W, true);
  });
  par_for(W, [&](int x) {
    if (hr == 0)
      return;
    std::vector<R> w(hr + 1), cd(hr), ci(hr), od(hr), oi(hr);
    for (int k = 0; k <= hr; ++k)
      w[k] = col_w[(size_t)k * W + x];
    for (int k = 0; k < hr; ++k)
    {
      cd[k] = rd[(size_t)k * W + x];
      ci[k] = ri[(size_t)k * W + x];
    }
    thomas_line<R>(hr, w.data(), 1, cd.data(), ci.data(), 1, lambda, od.data(), oi.data(), false);
    for (int k = 0; k < hr; ++k)
      dense[(size_t)k * W + x] = od[k] / oi[k];
  });
}

// ---------------------------------------------------------------------------
// Depth fusion: depth_fusion.cu:13-213 (fuse_transform, hole_filling,
// fuse_currentmap), with the reference's races resolved deterministically:
//  * z-buffer: the seed with the smallest transformed depth wins, ties to the
//    smallest pixel index (the reference keeps the nearer one but may give up
//    after 5 compare-and-swap retries or read a stale depth);
//  * hole filling: an empty pixel takes, among its non-empty 3x3 neighbours
//    with x, y in [2, W-1) x [2, H-1) (the pixels that propagate) of the
//    table after the z-buffer, the one whose seed is nearest (ties to the
//    smaller index) — one pass, no chains (the reference is first-writer-wins
//    and may chain);
//  * index 0 is the empty marker, so pixel (0, 0) never propagates (as in the
//    reference).
// contested[p] = 1 marks pixels whose reference result depends on thread
// timing: a z-buffer target hit by two or more seeds, or a pixel that is empty
// after the z-buffer with a non-empty pixel within Chebyshev distance 2.
//
// The seed transform is computed in float for both R (the seeds are float4
// in memory, as in the reference); R only sets the precision of the
// posterior update (fuse_currentmap).
template <typename R>
void fuse(const R *depth_in, const float *seeds_in, const float *T, const Cam &cam, int W, int H,
          R *depth_out, R *seeds_out, int *table_out, uint8_t *contested)
{
  const size_t N = (size_t)W * H;
  std::vector<float> tseed(seeds_in, seeds_in + 4 * N); // seeds after the write-back
  std::vector<int> target(N, -1);
  std::vector<float> tdepth(N, 0.0f);
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x)
    {
      const size_t idx = (size_t)y * W + x;
      const float a = seeds_in[4 * idx + 0], b = seeds_in[4 * idx + 1];
      const float mu = seeds_in[4 * idx + 2], s2 = seeds_in[4 * idx + 3];
      // is_badpoint (depth_fusion.cu:25-28)
      if ((double)a < 0.001 || (double)(a / (a + b)) < 0.45)
        continue;
      const float vx = ((float)x - cam.cx) / cam.fx;
      const float vy = ((float)y - cam.cy) / cam.fy;
      const float vz = 1.0f;
      const float inv_len = 1.0f / std::sqrt(vx * vx + vy * vy + vz * vz);
      const float px = vx * inv_len * mu, py = vy * inv_len * mu, pz = vz * inv_len * mu;
      const float qx = T[0] * px + T[1] * py + T[2] * pz + T[3];
      const float qy = T[4] * px + T[5] * py + T[6] * pz + T[7];
      const float qz = T[8] * px + T[9] * py + T[10] * pz + T[11];
      const float nd = std::sqrt(qx * qx + qy * qy + qz * qz);
      if ((double)nd <= 0.5)
        continue;
      const float nw = (float)((double)s2 + (double)nd * 0.01);
      const float u = cam.fx * qx / qz + cam.cx;
      const float v = cam.fy * qy / qz + cam.cy;
      const int tx = trunc_sat((double)u + 0.5), ty = trunc_sat((double)v + 0.5);
      if (tx >= W || tx < 0 || ty >= H || ty < 0)
        continue;
      tseed[4 * idx + 2] = nd;
      tseed[4 * idx + 3] = nw;
      tdepth[idx] = nd;
      target[idx] = ty * W + tx;
    }
  std::vector<int> table(N, 0), hits(N, 0);
  for (size_t idx = 0; idx < N; ++idx)
  {
    if (target[idx] < 0)
      continue;
    const int t = target[idx];
    hits[t] += 1;
    if (idx == 0)
      continue; // index 0 is the empty marker
    const int cur = table[t];
    if (cur == 0 || tdepth[idx] < tdepth[cur] || (tdepth[idx] == tdepth[cur] && (int)idx < cur))
      table[t] = (int)idx;
  }
  std::vector<int> filled(table);
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x)
    {
      const size_t c = (size_t)y * W + x;
      if (table[c] != 0)
        continue;
      int best = 0;
      for (int i = -1; i <= 1; ++i)
        for (int j = -1; j <= 1; ++j)
        {
          const int nx = x + j, ny = y + i;
          if (nx < 2 || nx >= W - 1 || ny < 2 || ny >= H - 1)
            continue;
          const int s = table[(size_t)ny * W + nx];
          if (s == 0)
            continue;
          if (best == 0 || tdepth[s] < tdepth[best] || (tdepth[s] == tdepth[best] && s < best))
            best = s;
        }
      filled[c] = best;
    }
  if (contested)
  {
    for (size_t c = 0; c < N; ++c)
      contested[c] = hits[c] >= 2 ? 1 : 0;
    for (int y = 0; y < H; ++y)
      for (int x = 0; x < W; ++x)
      {
        const size_t c = (size_t)y * W + x;
        if (table[c] != 0)
          continue;
        for (int i = -2; i <= 2 && !contested[c]; ++i)
          for (int j = -2; j <= 2; ++j)
          {
            const int nx = x + j, ny = y + i;
            if (nx < 0 || nx >= W || ny < 0 || ny >= H)
              continue;
            if (table[(size_t)ny * W + nx] != 0)
            {
              contested[c] = 1;
              break;
            }
          }
      }
  }
  for (size_t c = 0; c < N; ++c)
  {
    const R dep = depth_in[c];
    R unc = std::max((R)0.5f, (R)((double)dep * 0.2));
    unc *= unc;
    if (dep <= (R)0)
      unc = (R)1e9f;
    const int pre = filled[c];
    R a, b, mu, s2;
    if (pre > 0)
    {
      a = (R)tseed[4 * pre + 0];
      b = (R)tseed[4 * pre + 1];
      mu = (R)tseed[4 * pre + 2];
      s2 = (R)tseed[4 * pre + 3];
    }
    else
    {
      a = 10;
      b = 10;
      mu = dep;
      s2 = 2500;
    }
    if ((dep - mu) * (dep - mu) > unc + s2)
    {
      a = 10;
      b = 10;
      mu = dep;
      s2 = 2500;
    }
    const R new_sq = unc * s2 / (unc + s2);
    const R new_mu = (dep * s2 + mu * unc) / (unc + s2);
    const R var = unc + s2;
    const R pdf = std::exp(-(dep - mu) * (dep - mu) / ((R)2 * var)) *
                  ((R)1 / std::sqrt((R)(2.0 * M_PI * (double)var)));
    R c1 = (a / (a + b)) * pdf;
    R c2 = (b / (a + b)) * (R)1 / (R)50;
    const R norm = c1 + c2;
    c1 = c1 / norm;
    c2 = c2 / norm;
    const R f = c1 * ((a + 1) / (a + b + 1)) + c2 * (a / (a + b + 1));
    const R e = c1 * (((a + 1) * (a + 2)) / ((a + b + 1) * (a + b + 2))) +
                c2 * (a * (a + 1) / ((a + b + 1) * (a + b + 2)));
    const R mu_p = c1 * new_mu + c2 * mu;
    const R s2_p = c1 * (new_sq + new_mu * new_mu) + c2 * (s2 + mu * mu) - mu_p * mu_p;
    const R a_p = (e - f) / (f - e / f);
    const R b_p = a_p * ((R)1 - f) / f;
    depth_out[c] = ((double)(a / (a + b)) > 0.60) ? mu_p : (R)-1;
    seeds_out[4 * c + 0] = a_p;
    seeds_out[4 * c + 1] = b_p;
    seeds_out[4 * c + 2] = mu_p;
    seeds_out[4 * c + 3] = s2_p;
  }
  if (table_out)
    std::copy(filled.begin(), filled.end(), table_out);
}

} // namespace

// ---------------------------------------------------------------------------
// C entry points (ctypes).  Images are dense row-major, no padding.
extern "C" {

// Host threads used by the parallel loops (1 = scalar port).
void orc_set_threads(int n) { g_threads = n < 1 ? 1 : n; }
int orc_get_threads(void) { return g_threads; }

void orc_quadtree(const uint8_t *img, int w, int h, const orc_params *p, int *levels)
{
  quadtree_levels(img, w, h, p->qt_max_level, p->qt_min_level, p->qt_threshold, levels);
}

#define ORC_COST(NAME, R)                                                                     \
  void NAME(const uint8_t *ref, int w, int h, const int *levels, int nslots,                 \
            const uint8_t *const *slot_img, const float *T, float fx, float fy, float cx,     \
            float cy, const orc_params *p, R *cost, int *valid_cells)                         \
  {                                                                                           \
    Cam cam{fx, fy, cx, cy};                                                                  \
    cost_volume<R>(ref, w, h, levels, nslots, slot_img, T, cam, *p, cost, valid_cells);       \
  }
ORC_COST(orc_cost_f32, float)
ORC_COST(orc_cost_f64, double)

#define ORC_BP(NAME, R)                                                                       \
  void NAME(const R *cost, int W, int H, const int *levels, const orc_params *p, int *labels, \
            R *sparse, R *msg_out)                                                            \
  {                                                                                           \
    bp_extract<R>(cost, W, H, levels, *p, labels, sparse, msg_out);                           \
  }
ORC_BP(orc_bp_f32, float)
ORC_BP(orc_bp_f64, double)

#define ORC_UP(NAME, R)                                                                       \
  void NAME(const R *sparse, const uint8_t *img, int W, int H, const orc_params *p, R *dense) \
  {                                                                                           \
    upsample<R>(sparse, img, W, H, *p, dense);                                                \
  }
ORC_UP(orc_upsample_f32, float)
ORC_UP(orc_upsample_f64, double)

// differentiable path: soft BP readout and weighted upsampling, FP64
void orc_bp_soft_f64(const double *cost, int W, int H, const int *levels, const orc_params *p,
                     double tau, int *labels, double *sparse)
{
  bp_extract<double>(cost, W, H, levels, *p, labels, sparse, nullptr, tau);
}

void orc_upsample_w_f64(const double *sparse, const uint8_t *img, int W, int H,
                        const orc_params *p, const double *omega, double *dense)
{
  upsample<double>(sparse, img, W, H, *p, dense, omega);
}

void orc_upsample_weights_f32(const uint8_t *img, int W, int H, const orc_params *p,
                              float *row_w, float *col_w)
{
  upsample_weights<float>(img, W, H, *p, row_w, col_w);
}

#define ORC_FUSE(NAME, R)                                                                     \
  void NAME(const R *depth_in, const float *seeds_in, const float *T, float fx, float fy,     \
            float cx, float cy, int W, int H, R *depth_out, R *seeds_out, int *table_out,      \
            uint8_t *contested)                                                               \
  {                                                                                           \
    Cam cam{fx, fy, cx, cy};                                                                  \
    fuse<R>(depth_in, seeds_in, T, cam, W, H, depth_out, seeds_out, table_out, contested);    \
  }
ORC_FUSE(orc_fuse_f32, float)
ORC_FUSE(orc_fuse_f64, double)

// Point cloud of a depth map, Publisher::publishPointCloud
// (publisher.cpp:146-163): a pixel is kept unless its depth is below 0.1
// (the float compared as a double); its point is T * (n * depth) with n the
// unit ray ((x-cx)/fx, (y-cy)/fy, 1) scaled by 1/sqrt of its squared length
// (helper_math.h normalize with the host rsqrtf, :62-65,1364-1368), the rigid
// transform applied as a rotation, summed left to right, then the
// translation (se3.cuh:122-151).  Writes 4 floats (x, y, z, intensity) per
// point in row-major pixel order; returns the number of points.
int orc_point_cloud(const float *depth, const uint8_t *ref, int W, int H, float fx, float fy,
                    float cx, float cy, const float *T, float *xyzi)
{
  int n = 0;
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x)
    {
      const float d = depth[(size_t)y * W + x];
      if ((double)d < 0.1)
        continue;
      const float u = ((float)x - cx) / fx;
      const float v = ((float)y - cy) / fy;
      const float inv = 1.0f / std::sqrt(u * u + v * v + 1.0f);
      const float p[3] = {u * inv * d, v * inv * d, inv * d};
      float *o = xyzi + 4 * (size_t)n;
      for (int r = 0; r < 3; ++r)
      {
        const float rot = T[4 * r] * p[0] + T[4 * r + 1] * p[1] + T[4 * r + 2] * p[2];
        o[r] = rot + T[4 * r + 3];
      }
      o[3] = (float)ref[(size_t)y * W + x];
      ++n;
    }
  return n;
}

} // extern "C"
