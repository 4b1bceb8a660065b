// Semi-dense tracker: the LSD-style per-pixel inverse-depth seeds of the
// keyframe (lsd_semidense.cu, seed_init.cu; host sequence
// seed_matrix.cu:106-146,211-446), whose projection into the incoming frame
// is the sparse depth the upsampler starts from (the "debug image" the BP
// extraction then overwrites at quadtree-node pixels).
//
// One step per frame and stream, all streams of a batch in one launch per
// kernel (a block finds its stream through the block prefix).  Modes:
//   init   (first frame)  seeds from the incoming image's gradient
//   update                epipolar stereo update of every seed, hole
//                         filling, regularisation, projection into the frame
//   switch                update, then the seeds are propagated into the
//                         incoming frame, which becomes the keyframe
//
// Determinism.  The reference regularises and fills holes in place (a seed
// reads neighbours that other threads of the same launch may already have
// rewritten), resolves propagation collisions with at most five atomicCAS
// retries and lets the last writer win where two seeds project onto one
// pixel; its results depend on thread scheduling.  Here every neighbourhood
// kernel reads the state before the launch and writes a second buffer, a
// propagation collision keeps the nearest seed (largest inverse depth; ties:
// the larger source index) and a projection collision keeps the nearest
// depth (ties: the smaller source index), both through 64-bit atomicMin on a
// z-buffer key.  Everything else follows the reference kernels operation for
// operation, including their quirks: the search range of an update is always
// [0.01, 2.0] (lsd_semidense.cu:451-458 declares the narrowed bounds in an
// inner scope), hole filling reads the INCOMING image's gradient at the
// keyframe pixel (:349), a zero best score counts as a failed search.
//
// Arithmetic.  QM_ARITH_REFERENCE: the operators are the plain float ones of
// this fast-math translation unit and images are sampled by the texture unit
// with linear filtering (the reference's bindTexture), as the reference
// kernels do.  QM_ARITH_IEEE: every operation is an IEEE-rounded intrinsic
// and bilinear samples are computed in software with the texture unit's
// 8-bit weight arithmetic (sample() below), matching the CPU oracle bit for
// bit.  Both paths evaluate the same expression trees.
#include <climits>

#include "launch.h"
#include "semidense.h"

namespace qm
{

namespace
{

constexpr int kSdThreads = 256;
constexpr unsigned long long kSdEmpty = ~0ull;

// reference constants (stereo_parameter.cuh:1-41)
constexpr float kMinGrad = 5.0f;                       // MIN_GRAIDIENT
constexpr float kMinInvDepth = 0.01f;                  // MIN_INV_DEPTH
constexpr float kMaxInvDepth = 2.0f;                   // MAX_INV_DEPTH
constexpr double kVarMax = 4.0;                        // VARIANCE_MAX
constexpr float kMaxDiffConst = 40.0f * 40.0f;         // MAX_DIFF_CONSTANT
constexpr float kMaxDiffGradMult = 0.5f * 0.5f;        // MAX_DIFF_GRAD_MULT
constexpr float kRegDistVar = 0.075f * 0.075f;         // REG_DIST_VAR
constexpr float kValSumMinCreate = 24.0f;              // VAL_SUM_MIN_FOR_CREATE
constexpr float kValSumMinKeep = 24.0f;                // VAL_SUM_MIN_FOR_KEEP
constexpr float kValSumMinUnblacklist = 100.0f;        // VAL_SUM_MIN_FOR_UNBLACKLIST
constexpr float kMinBlacklist = -1.0f;                 // MIN_BLACKLIST
constexpr int kMaxSearch = 100;                        // MAX_SEARCH
constexpr float kMaxErrorStereo = 1300.0f;             // MAX_ERROR_STEREO
constexpr float kMinDistErrorStereo = 1.5f;            // MIN_DISTANCE_ERROR_STEREO
constexpr float kValidityInc = 5.0f;                   // VALIDITY_COUNTER_INC
constexpr float kValidityDec = 5.0f;                   // VALIDITY_COUNTER_DEC
constexpr float kValidityInitial = 5.0f;               // VALIDITY_COUNTER_INITIAL_OBSERVE
constexpr float kValidityMax = 5.0f;                   // VALIDITY_COUNTER_MAX
constexpr float kValidityMaxVariable = 250.0f;         // VALIDITY_COUNTER_MAX_VARIABLE
constexpr float kSuccVarIncFac = 1.01f;                // SUCC_VAR_INC_FAC
constexpr float kFailVarIncFac = 1.1f;                 // FAIL_VAR_INC_FAC

// ---------------------------------------------------------------------------
// Number type: Fl<false> uses the translation unit's float operators (the
// reference build's rounding and multiply-add contraction), Fl<true> the
// IEEE round-to-nearest intrinsics (never contracted).
template <bool I>
struct Fl
{
  float v;
  Fl() = default;
  __device__ __forceinline__ constexpr Fl(float x) : v(x) {}
};
template <bool I>
__device__ __forceinline__ Fl<I> operator+(Fl<I> a, Fl<I> b)
{
  return I ? __fadd_rn(a.v, b.v) : a.v + b.v;
}
template <bool I>
__device__ __forceinline__ Fl<I> operator-(Fl<I> a, Fl<I> b)
{
  return I ? __fsub_rn(a.v, b.v) : a.v - b.v;
}
template <bool I>
__device__ __forceinline__ Fl<I> operator*(Fl<I> a, Fl<I> b)
{
  return I ? __fmul_rn(a.v, b.v) : a.v * b.v;
}
template <bool I>
__device__ __forceinline__ Fl<I> operator/(Fl<I> a, Fl<I> b)
{
  return I ? __fdiv_rn(a.v, b.v) : a.v / b.v;
}
template <bool I>
__device__ __forceinline__ Fl<I> operator-(Fl<I> a)
{
  return Fl<I>(-a.v);
}
template <bool I>
__device__ __forceinline__ bool operator<(Fl<I> a, Fl<I> b) { return a.v < b.v; }
template <bool I>
__device__ __forceinline__ bool operator>(Fl<I> a, Fl<I> b) { return a.v > b.v; }
template <bool I>
__device__ __forceinline__ bool operator<=(Fl<I> a, Fl<I> b) { return a.v <= b.v; }
template <bool I>
__device__ __forceinline__ bool operator>=(Fl<I> a, Fl<I> b) { return a.v >= b.v; }
template <bool I>
__device__ __forceinline__ bool operator==(Fl<I> a, Fl<I> b) { return a.v == b.v; }
template <bool I>
__device__ __forceinline__ Fl<I> fsqrt(Fl<I> a)
{
  return I ? __fsqrt_rn(a.v) : sqrtf(a.v);
}

// (float)((double)v + c): the reference adds double literals to float
// texture coordinates and pixel positions
__device__ __forceinline__ float plus_d(float v, double c) { return (float)((double)v + c); }
__device__ __forceinline__ int trunc_plus_half(float v) { return (int)((double)v + 0.5); }

// ---------------------------------------------------------------------------
// The job of a block (block prefix over the streams of the step).
__device__ __forceinline__ const SdJob &sd_job(const SdBatch &B, int &lb)
{
  const int block = (int)blockIdx.x;
  if (B.jobs == nullptr)
  {
    lb = block;
    return B.one;
  }
  const int j = find_job(B.prefix, B.njobs, block);
  lb = block - __ldg(B.prefix + j);
  return B.jobs[j];
}

// pixel of this thread, false when outside the image
__device__ __forceinline__ bool sd_pixel(const SdJob &J, int lb, int &x, int &y)
{
  const int p = lb * kSdThreads + (int)threadIdx.x;
  if (p >= J.W * J.H)
    return false;
  y = p / J.W;
  x = p - y * J.W;
  return true;
}

// the reference's seed kernels touch 2 < x < W-3, 2 < y < H-3
__device__ __forceinline__ bool sd_interior(const SdJob &J, int x, int y)
{
  return !(x >= J.W - 3 || y >= J.H - 3 || x <= 2 || y <= 2);
}

__device__ __forceinline__ float texel(const float *img, size_t pitch, int x, int y)
{
  return img[(size_t)y * pitch + x];
}

// Bilinear sample at unnormalised (u, v) with clamp addressing.  Reference
// mode: the texture unit.  IEEE mode: the texture unit's arithmetic, as
// measured on a B200 (bit-identical over 26k samples): the fractional
// positions a, b are rounded to 8 bits (half up), the four corner weights
// (1-a)(1-b), a(1-b), (1-a)b, ab to 8 bits as well, the two diagonal ones
// half up and the two others half down (so that they sum to one), and the
// weighted sum of the texels is exact.
__device__ __forceinline__ float frac8(float t)
{
  const float f = floorf(t);
  return (t - f) >= 0.5f ? f + 1.0f : f; // t - f is exact
}
template <bool I>
__device__ __forceinline__ float sample(cudaTextureObject_t tex, const float *img, size_t pitch,
                                        int W, int H, float u, float v)
{
  if (!I)
    return tex2D<float>(tex, u, v);
  const float xb = __fsub_rn(u, 0.5f), yb = __fsub_rn(v, 0.5f);
  const float fx0 = floorf(xb), fy0 = floorf(yb);
  // 256 a and 256 b: integers in [0, 256]
  const float A = frac8(__fmul_rn(__fsub_rn(xb, fx0), 256.0f));
  const float B = frac8(__fmul_rn(__fsub_rn(yb, fy0), 256.0f));
  const float nA = 256.0f - A, nB = 256.0f - B;
  // 256 x the weights (products exact, the /256 and +-0.5 exact)
  const float w00 = floorf(__fadd_rn(__fmul_rn(__fmul_rn(nA, nB), 1.0f / 256.0f), 0.5f));
  const float w10 = ceilf(__fsub_rn(__fmul_rn(__fmul_rn(A, nB), 1.0f / 256.0f), 0.5f));
  const float w01 = ceilf(__fsub_rn(__fmul_rn(__fmul_rn(nA, B), 1.0f / 256.0f), 0.5f));
  const float w11 = floorf(__fadd_rn(__fmul_rn(__fmul_rn(A, B), 1.0f / 256.0f), 0.5f));
  const int i0 = __float2int_rz(fx0), j0 = __float2int_rz(fy0);
  const int xa = min(max(i0, 0), W - 1), xc = min(max(i0 == INT_MAX ? i0 : i0 + 1, 0), W - 1);
  const int ya = min(max(j0, 0), H - 1), yc = min(max(j0 == INT_MAX ? j0 : j0 + 1, 0), H - 1);
  // integer-valued terms below 2^16 each: the sum is exact
  float r = __fmul_rn(w00, texel(img, pitch, xa, ya));
  r = __fadd_rn(r, __fmul_rn(w10, texel(img, pitch, xc, ya)));
  r = __fadd_rn(r, __fmul_rn(w01, texel(img, pitch, xa, yc)));
  r = __fadd_rn(r, __fmul_rn(w11, texel(img, pitch, xc, yc)));
  return __fmul_rn(r, 1.0f / 256.0f);
}

// image gradient at an integer pixel (seed_init.cu:26-41): half central
// differences, exact for integer intensities
__device__ __forceinline__ float2 grad_at(const float *img, size_t pitch, int x, int y)
{
  const float r = texel(img, pitch, x + 1, y), l = texel(img, pitch, x - 1, y);
  const float d = texel(img, pitch, x, y + 1), u = texel(img, pitch, x, y - 1);
  return make_float2((float)((double)(r - l) / 2.0), (float)((double)(d - u) / 2.0));
}

template <bool I>
__device__ __forceinline__ Fl<I> dot2(float2 g)
{
  using F = Fl<I>;
  return F(g.x) * F(g.x) + F(g.y) * F(g.y);
}

struct Seed
{
  float4 t; // valid (> 0), blacklist, validity counter, unused
  float4 d; // idepth, variance, smooth idepth, smooth variance
};

__device__ __forceinline__ Seed load_seed(const SdJob &J, int sel, size_t o)
{
  const int b = J.cur ^ sel;
  return Seed{J.trk[b][o], J.dep[b][o]};
}
__device__ __forceinline__ void store_seed(const SdJob &J, int sel, size_t o, const Seed &s)
{
  const int b = J.cur ^ sel;
  J.trk[b][o] = s.t;
  J.dep[b][o] = s.d;
}
// DepthSeed::initialize (DepthSeed.cuh:15-26)
__device__ __forceinline__ Seed seed_init(float idepth, float var, float counter)
{
  return Seed{make_float4(1.0f, 0.0f, counter, 0.0f), make_float4(idepth, var, 1.0f, 4.0f)};
}
__device__ __forceinline__ bool valid(const Seed &s) { return s.t.x > 0.0f; }

// ---------------------------------------------------------------------------
// Conversion of the incoming u8 frame into the float image the textures
// read (the reference converts on the host, seed_matrix.cu:87).
__global__ void __launch_bounds__(kSdThreads) k_sd_convert(const __grid_constant__ SdBatch B)
{
  int lb, x, y;
  const SdJob &J = sd_job(B, lb);
  if (J.mode == kSdNone || !sd_pixel(J, lb, x, y))
    return;
  J.inc_f[(size_t)y * J.pitch + x] = (float)J.inc[(size_t)y * J.W + x];
}

// initialize_keyframe_kernel (lsd_semidense.cu:61-78)
__global__ void __launch_bounds__(kSdThreads) k_sd_init(const __grid_constant__ SdBatch B)
{
  int lb, x, y;
  const SdJob &J = sd_job(B, lb);
  if (J.mode != kSdInit || !sd_pixel(J, lb, x, y))
    return;
  const size_t o = (size_t)y * J.W + x;
  Seed s{make_float4(0.0f, 0.0f, 0.0f, 0.0f), make_float4(0.0f, 0.0f, 0.0f, 0.0f)};
  if (sd_interior(J, x, y))
  {
    // half-integer gradient components: the squared magnitude is exact in
    // either arithmetic
    const float2 g = grad_at(J.inc_f, J.pitch, x, y);
    if (!(__fadd_rn(__fmul_rn(g.x, g.x), __fmul_rn(g.y, g.y)) < kMinGrad * kMinGrad))
      s = Seed{make_float4(1.0f, 0.0f, 20.0f, 0.0f), make_float4(1.0f, 4.0f, 1.0f, 4.0f)};
  }
  store_seed(J, 0, o, s);
}

// Sum of the products of two five-sample residual sets, left to right.
template <bool I>
__device__ __forceinline__ Fl<I> residual_overlap(const Fl<I> (&a)[5], const Fl<I> (&b)[5])
{
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3] + a[4] * b[4];
}

// search_point (lsd_semidense.cu:517-754): epipolar line search of the
// keyframe pixel (x, y) in the incoming image.  Returns the match error or a
// negative failure code.  The operation order follows the reference's so
// that reference arithmetic rounds as it does; the residuals of the last even
// and the last odd step are kept apart because the sub-pixel step uses their
// overlap on both sides of the best match.
template <bool I>
__device__ float search_point(const SdJob &J, int x, int y, float2 epi, Fl<I> gradient_max,
                              Fl<I> my_gradient, Fl<I> min_idep, Fl<I> max_idep,
                              Fl<I> &result_idep, Fl<I> &result_var)
{
  using F = Fl<I>;
  const F fx(J.fx), fy(J.fy), cx(J.cx), cy(J.cy);
  const float *T = J.T;
  // five keyframe samples along the epipolar direction, centred on (x, y)
  F key_patch[5];
#pragma unroll
  for (int i = -2; i <= 2; i++)
  {
    const F px = F((float)x) + F((float)i) * F(epi.x);
    const F py = F((float)y) + F((float)i) * F(epi.y);
    key_patch[i + 2] = sample<I>(J.key_tex, J.key_f, J.pitch, J.W, J.H, plus_d(px.v, 0.5),
                                 plus_d(py.v, 0.5));
  }
  // the pixel's ray rotated into the incoming camera and projected (K R K^-1
  // p, homogeneous), and the projected translation (K t): a point at
  // inverse depth q lands at ray + q * shift
  const F kx = (F((float)x) - cx) / fx, ky = (F((float)y) - cy) / fy, kz(1.0f);
  const F rx = F(T[0]) * kx + F(T[1]) * ky + F(T[2]) * kz;
  const F ry = F(T[4]) * kx + F(T[5]) * ky + F(T[6]) * kz;
  const F rz = F(T[8]) * kx + F(T[9]) * ky + F(T[10]) * kz;
  const F tx(T[3]), ty(T[7]), tz(T[11]);
  const F ray_x = fx * rx + cx * rz, ray_y = fy * ry + cy * rz, ray_z = rz;
  const F shift_x = fx * tx + cx * tz, shift_y = fy * ty + cy * tz, shift_z = tz;
  const F nearx = ray_x + shift_x * max_idep, neary = ray_y + shift_y * max_idep,
          nearz = ray_z + shift_z * max_idep;
  const F farx = ray_x + shift_x * min_idep, fary = ray_y + shift_y * min_idep,
          farz = ray_z + shift_z * min_idep;
  F near_u = nearx / nearz, near_v = neary / nearz;
  F far_u = farx / farz, far_v = fary / farz;
  const F du = near_u - far_u, dv = near_v - far_v;
  F search_length = fsqrt(du * du + dv * dv);
  F dir_u = du / search_length, dir_v = dv / search_length;
  if ((double)search_length.v < 3.0)
  {
    near_u = near_u + dir_u * F(2.0f);
    near_v = near_v + dir_v * F(2.0f);
    far_u = far_u - dir_u * F(2.0f);
    far_v = far_v - dir_v * F(2.0f);
    search_length = F(plus_d(search_length.v, 4.0));
  }
  if (far_u.v <= 1.0f || far_v.v <= 1.0f || far_u.v >= (float)(J.W - 2) ||
      far_v.v >= (float)(J.H - 2))
    return -1.0f;

  // five incoming-image samples ending at the current step, oldest first
  F line_patch[5];
#pragma unroll
  for (int i = -2; i <= 1; i++)
  {
    const F px = far_u + F((float)i) * dir_u, py = far_v + F((float)i) * dir_v;
    line_patch[i + 2] = sample<I>(J.inc_tex, J.inc_f, J.pitch, J.W, J.H, plus_d(px.v, 0.5),
                                  plus_d(py.v, 0.5));
  }
  F best_step(-1.0f), best_score(1e9f), score_before_best(1e9f), score_after_best(1e9f);
  bool last_is_best = false;
  F overlap_before(NAN), overlap_after(NAN);
  F res_even[5], res_odd[5];
#pragma unroll
  for (int j = 0; j < 5; ++j)
    res_even[j] = res_odd[j] = F(NAN);
  F second_best_score(1e9f), second_best_step(-1.0f);
  F prev_score(1e9f), score(1e9f);
  // the sample of step s + 1 is fetched while step s is scored (sampling is
  // a pure function of its coordinates and clamps, so the fetch past the last
  // step is harmless)
  auto fetch = [&](int step) {
    const F sx = far_u + F((float)step) * dir_u, sy = far_v + F((float)step) * dir_v;
    return sample<I>(J.inc_tex, J.inc_f, J.pitch, J.W, J.H,
                     (float)((double)sx.v + 2.0 * (double)dir_u.v + 0.5),
                     (float)((double)sy.v + 2.0 * (double)dir_v.v + 0.5));
  };
  F next = fetch(0);
  for (int step = 0; (float)step <= search_length.v && step <= kMaxSearch; step += 1)
  {
    prev_score = score;
    score = F(0.0f);
    const F sx = far_u + F((float)step) * dir_u, sy = far_v + F((float)step) * dir_v;
    if (sx.v <= 1.0f || sx.v >= (float)(J.W - 1) || sy.v <= 1.0f || sy.v >= (float)(J.H - 1))
      break;
    line_patch[4] = next;
    next = fetch(step + 1);
    // squared residuals, newest sample first
    if (step % 2 == 0)
    {
#pragma unroll
      for (int j = 0; j < 5; ++j)
      {
        res_even[j] = line_patch[4 - j] - key_patch[4 - j];
        score = score + res_even[j] * res_even[j];
      }
    }
    else
    {
#pragma unroll
      for (int j = 0; j < 5; ++j)
      {
        res_odd[j] = line_patch[4 - j] - key_patch[4 - j];
        score = score + res_odd[j] * res_odd[j];
      }
    }
    if (last_is_best)
    {
      score_after_best = score;
      overlap_after = residual_overlap<I>(res_even, res_odd);
      last_is_best = false;
    }
    if (score < best_score)
    {
      second_best_score = best_score;
      second_best_step = best_step;
      best_score = score;
      best_step = F((float)step);
      score_before_best = prev_score;
      overlap_before = residual_overlap<I>(res_even, res_odd);
      overlap_after = F(-1.0f);
      score_after_best = F(1e9f);
      last_is_best = true;
    }
    else if (score < second_best_score)
    {
      second_best_score = score;
      second_best_step = F((float)step);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j)
      line_patch[j] = line_patch[j + 1];
  }

  if (best_score > F(4.0f * kMaxErrorStereo))
    return -3.0f;
  if (fabsf((second_best_step - best_step).v) > 1.0f &&
      F(kMinDistErrorStereo) * best_score > second_best_score)
    return -2.0f;

  // sub-pixel refinement from the score slopes on either side of the best
  // step
  F best_match_sub = best_step;
  bool did_subpixel = false;
  {
    const F slope_before_out = -(score_before_best - overlap_before);
    const F slope_before_in = best_score - overlap_before;
    const F slope_after_in = -(best_score - overlap_after);
    const F slope_after_out = score_after_best - overlap_after;
    bool use_after = false, use_before = false;
    if ((slope_before_out.v < 0.0f) ^ (slope_before_in.v < 0.0f))
    {
      if (!((slope_after_out.v < 0.0f) ^ (slope_after_in.v < 0.0f)))
        use_before = true;
    }
    else if ((slope_after_out.v < 0.0f) ^ (slope_after_in.v < 0.0f))
      use_after = true;
    if (use_before)
    {
      const F d = slope_before_in / (slope_before_in - slope_before_out);
      best_match_sub = best_match_sub - d;
      best_score = best_score - F(2.0f) * d * slope_before_in -
                   (slope_before_out - slope_before_in) * d * d;
      did_subpixel = true;
    }
    else if (use_after)
    {
      const F d = slope_after_in / (slope_after_in - slope_after_out);
      best_match_sub = best_match_sub - d;
      best_score = best_score + F(2.0f) * d * slope_after_in +
                   (slope_after_out - slope_after_in) * d * d;
      did_subpixel = true;
    }
  }

  F grad_along_line(0.0f);
#pragma unroll
  for (int i = 1; i < 5; i++)
    grad_along_line =
        grad_along_line + (key_patch[i] - key_patch[i - 1]) * (key_patch[i] - key_patch[i - 1]);
  if (best_score > F(kMaxErrorStereo) + fsqrt(grad_along_line) * F(20.0f))
    return -3.0f;

  // inverse depth of the match from the coordinate that moves most along the
  // line, and its derivative with respect to that coordinate
  F best_idepth, alpha;
  if (dir_u * dir_u > dir_v * dir_v)
  {
    const F best_u = far_u + best_match_sub * dir_u;
    best_idepth = (best_u * ray_z - ray_x) / (shift_x - best_u * shift_z);
    alpha = (ray_z * shift_x - shift_z * ray_x) /
            ((shift_x - best_u * shift_z) * (shift_x - best_u * shift_z));
  }
  else
  {
    const F best_v = far_v + best_match_sub * dir_v;
    best_idepth = (best_v * ray_z - ray_y) / (shift_y - best_v * shift_z);
    alpha = (ray_z * shift_y - shift_z * ray_y) /
            ((shift_y - best_v * shift_z) * (shift_y - best_v * shift_z));
  }
  best_idepth = (double)best_idepth.v < 0.01 ? F(kMinInvDepth) : best_idepth;
  best_idepth = (double)best_idepth.v > 2.0 ? F(kMaxInvDepth) : best_idepth;

  const F photo = F(4.0f * 4.0f) / my_gradient / my_gradient;
  const F geo = F(0.25f) * gradient_max * gradient_max / (my_gradient * my_gradient);
  const double sub = did_subpixel ? 0.05 : 0.5;
  result_var = F((float)((double)(alpha * alpha).v * (sub + (double)geo.v + (double)photo.v)));
  result_idep = best_idepth;
  return best_score.v;
}

// update_keyframe_kernel (lsd_semidense.cu:400-515): one stereo observation
// per seed; reads and writes only its own seed.
// 4 blocks per SM (at most 64 registers instead of 86 / 102, i.e. 2 blocks):
// the search loop is latency-bound, and the extra resident warps outweigh
// the spilled values (tracker per stream and frame at 752x480: 0.171 ms at
// 2 blocks, 0.144 at 3, 0.127 at 4, 0.125 at 5)
template <bool I>
__global__ void __launch_bounds__(kSdThreads, 4) k_sd_update(const __grid_constant__ SdBatch B)
{
  using F = Fl<I>;
  int lb, x, y;
  const SdJob &J = sd_job(B, lb);
  if (J.mode < kSdUpdate || !sd_pixel(J, lb, x, y) || !sd_interior(J, x, y))
    return;
  const float2 g = grad_at(J.key_f, J.pitch, x, y);
  const F gradient_max = fsqrt(dot2<I>(g));
  if (gradient_max < F(kMinGrad))
    return;
  const size_t o = (size_t)y * J.W + x;
  Seed s = load_seed(J, 0, o);
  if (s.t.y < kMinBlacklist)
    return;
  const bool first_observe = !valid(s);
  const float *T = J.T;
  // translation of the inverse of T (se3.cuh:91-107)
  const F itx = -F(T[0]) * F(T[3]) - F(T[4]) * F(T[7]) - F(T[8]) * F(T[11]);
  const F ity = -F(T[1]) * F(T[3]) - F(T[5]) * F(T[7]) - F(T[9]) * F(T[11]);
  const F itz = -F(T[2]) * F(T[3]) - F(T[6]) * F(T[7]) - F(T[10]) * F(T[11]);
  F ex = -F(J.fx) * itx + itz * (F((float)x) - F(J.cx));
  F ey = -F(J.fy) * ity + itz * (F((float)y) - F(J.cy));
  const F epi_length = fsqrt(ex * ex + ey * ey);
  if ((double)epi_length.v < 1.0)
    return;
  ex = ex / epi_length;
  ey = ey / epi_length;
  const F gae = F(fabsf((ex * F(g.x) + ey * F(g.y)).v));
  if ((double)gae.v < 2.0)
    return;
  if ((double)(gae / gradient_max).v < 0.3)
    return;

  F result_idep(0.0f), result_var(0.0f);
  const float err = search_point<I>(J, x, y, make_float2(ex.v, ey.v), gradient_max, gae,
                                    F(kMinInvDepth), F(kMaxInvDepth), result_idep, result_var);
  const F diff = result_idep - F(s.d.z);
  if (first_observe)
  {
    if (err == -3.0f || err == -2.0f)
      s.t.y = s.t.y - 1.0f;
    if (err > 0.0f && (double)result_var.v < kVarMax)
      s = seed_init(result_idep.v, result_var.v, kValidityInitial);
  }
  else
  {
    if (err == -2.0f)
    {
      s.t.z = s.t.z - kValidityDec;
      s.t.z = s.t.z < 0.0f ? 0.0f : s.t.z;
      s.d.y = (F(s.d.y) * F(kFailVarIncFac)).v;
      if ((double)s.d.y > kVarMax)
      {
        s.t.x = -1.0f;
        s.t.y = s.t.y - 1.0f;
      }
    }
    else if (err == -1.0f || err == -3.0f || err == -4.0f)
      return;
    else if (diff * diff > result_var + F(s.d.w))
    {
      s.d.y = (F(s.d.y) * F(kFailVarIncFac)).v;
      if ((double)s.d.y > kVarMax)
        s.t.x = -1.0f;
    }
    else
    {
      const F inc_var = F(s.d.y) * F(kSuccVarIncFac);
      const F new_var = (inc_var * result_var) / (inc_var + result_var);
      const F new_idepth = (F(s.d.x) * result_var + result_idep * inc_var) / (inc_var + result_var);
      if (new_var < F(s.d.y))
        s.d.y = new_var.v;
      s.d.x = new_idepth.v;
      s.t.z = s.t.z + kValidityInc;
      const F max_valid = F(kValidityMax) + gradient_max * F(kValidityMaxVariable) / F(255.0f);
      s.t.z = F(s.t.z) > max_valid ? max_valid.v : s.t.z;
    }
  }
  store_seed(J, 0, o, s);
}

// regulizeDepth_FillHoles_kernel (lsd_semidense.cu:342-383) from buffer
// `src` into the other buffer; the gradient test reads the incoming image.
template <bool I>
__global__ void __launch_bounds__(kSdThreads)
    k_sd_fill(const __grid_constant__ SdBatch B, int src, int min_mode)
{
  using F = Fl<I>;
  int lb, x, y;
  const SdJob &J = sd_job(B, lb);
  if (J.mode < min_mode || !sd_pixel(J, lb, x, y))
    return;
  const size_t o = (size_t)y * J.W + x;
  Seed s = load_seed(J, src, o);
  if (sd_interior(J, x, y) && !valid(s) &&
      !(dot2<I>(grad_at(J.inc_f, J.pitch, x, y)) < F(kMinGrad * kMinGrad)))
  {
    F sum_idepth(0.0f), sum_ivar(0.0f), sum_valid(0.0f);
    for (int j = -2; j <= 2; j++)
      for (int i = -2; i <= 2; i++)
      {
        const Seed n = load_seed(J, src, o + (long)j * J.W + i);
        if (valid(n))
        {
          sum_valid = sum_valid + F(n.t.z);
          const F w = F(1.0f) / F(n.d.y);
          sum_idepth = sum_idepth + F(n.d.x) * w;
          sum_ivar = sum_ivar + w;
        }
      }
    const bool create = (sum_valid > F(kValSumMinUnblacklist)) ||
                        (s.t.y >= kMinBlacklist && sum_valid > F(kValSumMinCreate));
    if (create)
      s = seed_init((sum_idepth / sum_ivar).v, (F(1.0f) / sum_ivar).v, 0.0f);
  }
  store_seed(J, src ^ 1, o, s);
}

// regulizeDepth_kernel (lsd_semidense.cu:284-341) from buffer `src` into
// the other buffer
template <bool I>
__global__ void __launch_bounds__(kSdThreads)
    k_sd_regularize(const __grid_constant__ SdBatch B, int src, int remove_occlusions,
                    int min_mode)
{
  using F = Fl<I>;
  int lb, x, y;
  const SdJob &J = sd_job(B, lb);
  if (J.mode < min_mode || !sd_pixel(J, lb, x, y))
    return;
  const size_t o = (size_t)y * J.W + x;
  Seed s = load_seed(J, src, o);
  if (sd_interior(J, x, y) && valid(s))
  {
    F sum_idepth(0.0f), sum_ivar(0.0f), sum_valid(0.0f);
    int occlusion = 0, not_occlusion = 0;
    for (int j = -2; j <= 2; j++)
      for (int i = -2; i <= 2; i++)
      {
        const Seed n = load_seed(J, src, o + (long)j * J.W + i);
        if (!valid(n))
          continue;
        const F diff = F(s.d.x) - F(n.d.x);
        if (diff * diff > F(s.d.y) + F(n.d.y))
        {
          if (s.d.x < n.d.x)
            occlusion++;
          continue;
        }
        sum_valid = sum_valid + F(n.t.z);
        not_occlusion++;
        const F spatial = F(kRegDistVar) * F((float)(i * i + j * j));
        const F ivar = F(1.0f) / (F(n.d.y) + spatial);
        sum_idepth = sum_idepth + ivar * F(n.d.x);
        sum_ivar = sum_ivar + ivar;
      }
    if (sum_valid < F(kValSumMinKeep))
      s.t.x = -1.0f;
    if (remove_occlusions && occlusion > not_occlusion)
      s.t.x = -1.0f;
    s.d.z = (sum_idepth / sum_ivar).v;
    s.d.w = (F(1.0f) / sum_ivar).v;
  }
  store_seed(J, src ^ 1, o, s);
}

// Projection of the seed at keyframe pixel (x, y) into the incoming frame
// with the reference's gates (depth_project_kernel :180-235 and
// propogate_keyframe_kernel :100-146 share them).  Returns false when a gate
// rejects it.
template <bool I>
__device__ __forceinline__ bool project_seed(const SdJob &J, int x, int y, float sidepth,
                                             Fl<I> &px, Fl<I> &py, Fl<I> &pz, Fl<I> &new_idepth,
                                             int &nx, int &ny)
{
  using F = Fl<I>;
  const F fx(J.fx), fy(J.fy), cx(J.cx), cy(J.cy);
  F kx = (F((float)x) - cx) / fx, ky = (F((float)y) - cy) / fy, kz(1.0f);
  kx = kx / F(sidepth);
  ky = ky / F(sidepth);
  kz = kz / F(sidepth);
  const float *T = J.T;
  px = F(T[0]) * kx + F(T[1]) * ky + F(T[2]) * kz + F(T[3]);
  py = F(T[4]) * kx + F(T[5]) * ky + F(T[6]) * kz + F(T[7]);
  pz = F(T[8]) * kx + F(T[9]) * ky + F(T[10]) * kz + F(T[11]);
  new_idepth = F(1.0f) / pz;
  nx = trunc_plus_half((px * new_idepth * fx + cx).v);
  ny = trunc_plus_half((py * new_idepth * fy + cy).v);
  if (nx <= 2 || nx >= J.W - 3 || ny <= 2 || ny >= J.H - 3)
    return false;
  const float2 g = grad_at(J.inc_f, J.pitch, nx, ny);
  const F g2 = dot2<I>(g);
  if (g2 < F(kMinGrad * kMinGrad))
    return false;
  const F old_color(texel(J.key_f, J.pitch, x, y));
  const F new_color(texel(J.inc_f, J.pitch, nx, ny));
  const F diff = old_color - new_color;
  return !(diff * diff > (F(kMaxDiffConst) + F(kMaxDiffGradMult) * g2));
}

// depth_project_kernel (lsd_semidense.cu:180-235): nearest-wins z-buffer of
// the projected depths of confident seeds
template <bool I>
__global__ void __launch_bounds__(kSdThreads) k_sd_project(const __grid_constant__ SdBatch B)
{
  using F = Fl<I>;
  int lb, x, y;
  const SdJob &J = sd_job(B, lb);
  if (J.mode < kSdUpdate || !sd_pixel(J, lb, x, y) || !sd_interior(J, x, y))
    return;
  const size_t o = (size_t)y * J.W + x;
  const Seed s = load_seed(J, 0, o);
  if (!valid(s) || s.t.z < 20.0f)
    return;
  F px, py, pz, nid;
  int nx, ny;
  if (!project_seed<I>(J, x, y, s.d.z, px, py, pz, nid, nx, ny))
    return;
  const F depth = fsqrt(px * px + py * py + pz * pz);
  if (depth.v != depth.v || (double)s.d.w > 0.02)
    return;
  const unsigned long long key =
      ((unsigned long long)__float_as_uint(depth.v) << 32) | (unsigned)o;
  atomicMin(J.zkey + (size_t)ny * J.W + nx, key);
}

// debug image of the step: the winning projected depth or 0; resets the
// z-buffer
__global__ void __launch_bounds__(kSdThreads) k_sd_resolve(const __grid_constant__ SdBatch B)
{
  int lb, x, y;
  const SdJob &J = sd_job(B, lb);
  if (J.mode == kSdNone || !sd_pixel(J, lb, x, y))
    return;
  const size_t o = (size_t)y * J.W + x;
  const unsigned long long key = J.zkey[o];
  J.debug[o] = key == kSdEmpty ? 0.0f : __uint_as_float((unsigned)(key >> 32));
  if (key != kSdEmpty)
    J.zkey[o] = kSdEmpty;
}

// order-preserving unsigned image of a float (larger float, larger key)
__device__ __forceinline__ unsigned ordered(float f)
{
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// propogate_keyframe_kernel (lsd_semidense.cu:100-178): every seed that
// survives the gates bids for its pixel in the incoming frame; the largest
// inverse depth wins (ties: the larger source index)
template <bool I>
__global__ void __launch_bounds__(kSdThreads) k_sd_propagate(const __grid_constant__ SdBatch B)
{
  using F = Fl<I>;
  int lb, x, y;
  const SdJob &J = sd_job(B, lb);
  if (J.mode != kSdSwitch || !sd_pixel(J, lb, x, y) || !sd_interior(J, x, y))
    return;
  const size_t o = (size_t)y * J.W + x;
  const Seed s = load_seed(J, 0, o);
  if (!valid(s))
    return;
  F px, py, pz, nid;
  int nx, ny;
  if (!project_seed<I>(J, x, y, s.d.z, px, py, pz, nid, nx, ny))
    return;
  const unsigned long long key = ~(((unsigned long long)ordered(nid.v) << 32) | (unsigned)o);
  atomicMin(J.zkey + (size_t)ny * J.W + nx, key);
}

// initialize_keyframe_kernel (lsd_semidense.cu:80-98): the new keyframe's
// seeds from the winning bids (into the other buffer); resets the z-buffer
template <bool I>
__global__ void __launch_bounds__(kSdThreads) k_sd_adopt(const __grid_constant__ SdBatch B)
{
  using F = Fl<I>;
  int lb, x, y;
  const SdJob &J = sd_job(B, lb);
  if (J.mode != kSdSwitch || !sd_pixel(J, lb, x, y))
    return;
  const size_t o = (size_t)y * J.W + x;
  const unsigned long long key = J.zkey[o];
  Seed n{make_float4(0.0f, 0.0f, 0.0f, 0.0f), make_float4(0.0f, 0.0f, 0.0f, 0.0f)};
  if (key != kSdEmpty)
  {
    J.zkey[o] = kSdEmpty;
    if (sd_interior(J, x, y))
    {
      const unsigned src = (unsigned)(~key & 0xffffffffull);
      const int sx = (int)(src % (unsigned)J.W), sy = (int)(src / (unsigned)J.W);
      const Seed s = load_seed(J, 0, src);
      F px, py, pz, nid;
      int nx, ny;
      project_seed<I>(J, sx, sy, s.d.z, px, py, pz, nid, nx, ny);
      // the new variance: (new_idepth / smooth_idepth)^4 * smooth variance
      F r = nid / F(s.d.z);
      r = r * r;
      r = r * r;
      const F new_var = r * F(s.d.w);
      n = seed_init(nid.v, new_var.v, s.t.z);
    }
  }
  store_seed(J, 1, o, n);
}

__global__ void __launch_bounds__(kSdThreads)
    k_u8_to_f32(const uint8_t *src, int W, int H, float *dst, size_t pitch)
{
  const long p = (long)blockIdx.x * kSdThreads + threadIdx.x;
  if (p >= (long)W * H)
    return;
  const int y = (int)(p / W), x = (int)(p - (long)y * W);
  dst[(size_t)y * pitch + x] = (float)src[p];
}

template <bool I>
void sd_sequence(const SdBatch &B, int blocks, cudaStream_t s)
{
  k_sd_convert<<<blocks, kSdThreads, 0, s>>>(B);
  k_sd_init<<<blocks, kSdThreads, 0, s>>>(B);
  // update_keyframe (seed_matrix.cu:401-446): stereo update, hole filling,
  // regularisation, projection into the incoming frame
  k_sd_update<I><<<blocks, kSdThreads, 0, s>>>(B);
  k_sd_fill<I><<<blocks, kSdThreads, 0, s>>>(B, 0, kSdUpdate);
  k_sd_regularize<I><<<blocks, kSdThreads, 0, s>>>(B, 1, 0, kSdUpdate);
  k_sd_project<I><<<blocks, kSdThreads, 0, s>>>(B);
  k_sd_resolve<<<blocks, kSdThreads, 0, s>>>(B);
  // create_new_keyframe (seed_matrix.cu:246-304): propagation into the
  // incoming frame, then regularisation with occlusion removal, hole filling
  // and regularisation
  k_sd_propagate<I><<<blocks, kSdThreads, 0, s>>>(B);
  k_sd_adopt<I><<<blocks, kSdThreads, 0, s>>>(B);
  k_sd_regularize<I><<<blocks, kSdThreads, 0, s>>>(B, 1, 1, kSdSwitch);
  k_sd_fill<I><<<blocks, kSdThreads, 0, s>>>(B, 0, kSdSwitch);
  k_sd_regularize<I><<<blocks, kSdThreads, 0, s>>>(B, 1, 0, kSdSwitch);
}

} // namespace

int sd_blocks(int W, int H) { return (W * H + kSdThreads - 1) / kSdThreads; }

void launch_u8_to_f32(const uint8_t *src, int W, int H, float *dst, size_t pitch,
                      cudaStream_t s)
{
  k_u8_to_f32<<<sd_blocks(W, H), kSdThreads, 0, s>>>(src, W, H, dst, pitch);
}

size_t sd_texture_pitch(int W)
{
  int dev = 0, align = 32;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&align, cudaDevAttrTexturePitchAlignment, dev);
  if (align < 4)
    align = 4;
  const size_t bytes = ((size_t)W * sizeof(float) + align - 1) / align * align;
  return bytes / sizeof(float);
}

cudaTextureObject_t sd_make_texture(const float *img, int W, int H, size_t pitch)
{
  cudaResourceDesc res = {};
  res.resType = cudaResourceTypePitch2D;
  res.res.pitch2D.devPtr = const_cast<float *>(img);
  res.res.pitch2D.desc = cudaCreateChannelDesc<float>();
  res.res.pitch2D.width = W;
  res.res.pitch2D.height = H;
  res.res.pitch2D.pitchInBytes = pitch * sizeof(float);
  cudaTextureDesc td = {};
  td.addressMode[0] = cudaAddressModeClamp;
  td.addressMode[1] = cudaAddressModeClamp;
  td.filterMode = cudaFilterModeLinear;
  td.readMode = cudaReadModeElementType;
  td.normalizedCoords = 0;
  cudaTextureObject_t t = 0;
  if (cudaCreateTextureObject(&t, &res, &td, nullptr) != cudaSuccess)
    return 0;
  return t;
}

int launch_semidense(const SdBatch &B, int blocks, int ieee, cudaStream_t s)
{
  if (blocks <= 0)
    return 0;
  if (ieee)
    sd_sequence<true>(B, blocks, s);
  else
    sd_sequence<false>(B, blocks, s);
  return 12;
}

} // namespace qm
