// extern "C" entry points of libqm_b200.so (declared in include/qm_capi.h).
// Every entry point catches all exceptions and returns a status code; the
// message is kept per thread for qm_last_error().
#include <algorithm>
#include <cstring>
#include <new>

#include "semidense.h"
#include "streams.h"

namespace qm
{
namespace stage
{
Batch single(const JobDesc &J);
int run_range(const Batch &B, const Shape &s, const qm_params &p, int first, int last,
              cudaStream_t stream);
int first_of(const char *name, int L);
int last_of(const char *name, int L);
} // namespace stage
} // namespace qm

struct qm_depthmap
{
  std::unique_ptr<qm::StreamSet> set;
  float fx, fy, cx, cy;
  int width, height;
};

struct qm_batch
{
  std::unique_ptr<qm::StreamSet> set;
};

namespace
{

using qm::CudaError;

template <class F>
int guarded(F &&f)
{
  try
  {
    f();
    qm::set_error("");
    return QM_OK;
  }
  catch (const CudaError &e)
  {
    qm::set_error(e.msg);
    return e.status;
  }
  catch (const std::bad_alloc &)
  {
    qm::set_error("host allocation failed");
    return QM_ERR_NO_MEMORY;
  }
  catch (const std::exception &e)
  {
    qm::set_error(e.what());
    return QM_ERR_CUDA;
  }
  catch (...)
  {
    qm::set_error("unknown error");
    return QM_ERR_CUDA;
  }
}

void require(bool ok, const char *msg)
{
  if (!ok)
    throw CudaError{QM_ERR_INVALID_ARG, msg};
}

qm_params params_or_default(const qm_params *p)
{
  qm_params q;
  if (p)
    q = *p;
  else
    qm_params_default(&q);
  const std::string err = qm::validate(q);
  require(err.empty(), err.c_str());
  return q;
}

cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

size_t bp_workspace(int W, int H, const qm_params &p)
{
  size_t o = 0;
  int w = W / 4, h = H / 4;
  for (int l = 0; l < p.bp_levels; ++l)
  {
    const size_t n = (size_t)w * h * p.num_hyp * sizeof(float);
    if (l > 0)
      o += align256(n);
    o += 4 * align256(n);
    w = (w + 1) / 2;
    h = (h + 1) / 2;
  }
  return o;
}

// the row-pass result (smoothed depth, smoothed indicator) per pixel
size_t upsample_workspace(int W, int H) { return align256((size_t)W * H * sizeof(float2)); }

size_t fuse_workspace(int W, int H) { return align256((size_t)W * H * 8); }

void check_stage_size(int W, int H)
{
  require(W >= 8 && H >= 8 && W <= 16384 && H <= 16384, "image size must be within [8, 16384]");
}

qm::JobDesc base_desc(int W, int H, const qm_params &p)
{
  qm::JobDesc J;
  std::memset(&J, 0, sizeof(J));
  J.W = W;
  J.H = H;
  J.D = p.num_hyp;
  J.F = 1;
  J.cw = W / 4;
  J.ch = H / 4;
  J.min_inv = p.min_inv_depth;
  J.step = p.inv_depth_step;
  J.nlev = p.bp_levels;
  return J;
}

qm::Shape stage_shape(int W, int H, const qm_params &p, int F, const qm_camera *cam)
{
  qm::Shape s;
  s.W = W;
  s.H = H;
  s.D = p.num_hyp;
  s.F = F;
  s.cam = cam ? qm::Cam{cam->fx, cam->fy, cam->cx, cam->cy} : qm::Cam{1, 1, 0, 0};
  return s;
}

void run_stage(const qm::JobDesc &J, const qm_params &p, const qm::Shape &s, const char *name,
               void *stream, const qm::SlotInline *slots = nullptr)
{
  qm::Batch B = qm::stage::single(J);
  if (slots)
    B.slots = *slots;
  qm::stage::run_range(B, s, p, qm::stage::first_of(name, p.bp_levels),
                       qm::stage::last_of(name, p.bp_levels), as_stream(stream));
}

// Workspace of the soft BP: the BP workspace of qm_bp_extract (pyramid data
// and messages of every level), the message states of one level's half-sweeps
// for the adjoint (sized for the largest level: iterations + 1 states), and
// two adjoint buffers of the level-0 size.
struct SoftLayout
{
  size_t bp = 0, hist = 0, dir = 0, total = 0;
};

SoftLayout soft_layout(int W, int H, const qm_params &p)
{
  SoftLayout L;
  L.bp = bp_workspace(W, H, p);
  int w = W / 4, h = H / 4;
  L.dir = align256((size_t)w * h * p.num_hyp * sizeof(float));
  for (int l = 0; l < p.bp_levels; ++l)
  {
    const size_t n = align256((size_t)w * h * p.num_hyp * sizeof(float));
    L.hist = std::max(L.hist, (size_t)(p.bp_iters[l] + 1) * 4 * n);
    w = (w + 1) / 2;
    h = (h + 1) / 2;
  }
  L.total = L.bp + L.hist + 2 * 4 * L.dir;
  return L;
}

int cdiv_i(long a, long b) { return (int)((a + b - 1) / b); }

// Soft BP of one keyframe over a caller workspace (see SoftLayout).
struct SoftBp
{
  qm::JobDesc J;
  SoftLayout lay;
  char *hist = nullptr, *adj[2] = {nullptr, nullptr};

  SoftBp(const float *cost, int W, int H, const uint8_t *levels, const qm_params &q, void *ws,
         size_t bytes)
  {
    lay = soft_layout(W, H, q);
    if (!ws || bytes < lay.total)
      throw CudaError{QM_ERR_WORKSPACE, "soft BP workspace too small"};
    require(((uintptr_t)cost | (uintptr_t)ws) % 16 == 0,
            "cost and workspace must be 16-byte aligned");
    J = base_desc(W, H, q);
    J.levels = const_cast<uint8_t *>(levels);
    char *b = (char *)ws;
    size_t o = 0;
    int w = W / 4, h = H / 4;
    for (int l = 0; l < q.bp_levels; ++l)
    {
      const size_t n = (size_t)w * h * q.num_hyp * sizeof(float);
      J.lv[l].w = w;
      J.lv[l].h = h;
      if (l == 0)
        J.lv[l].data = const_cast<float *>(cost);
      else
      {
        J.lv[l].data = (float *)(b + o);
        o += align256(n);
      }
      for (int m = 0; m < 4; ++m)
      {
        J.lv[l].msg[m] = (float *)(b + o);
        o += align256(n);
      }
      w = (w + 1) / 2;
      h = (h + 1) / 2;
    }
    hist = b + lay.bp;
    adj[0] = hist + lay.hist;
    adj[1] = adj[0] + 4 * lay.dir;
  }

  qm::DiffBp level_args(int l, const qm_params &q, float tau) const
  {
    qm::DiffBp a;
    std::memset(&a, 0, sizeof(a));
    a.W = J.W;
    a.H = J.H;
    a.D = q.num_hyp;
    a.w = J.lv[l].w;
    a.h = J.lv[l].h;
    a.level = l;
    a.qt_max = q.qt_max_level;
    a.levels = J.levels;
    a.data = J.lv[l].data;
    for (int m = 0; m < 4; ++m)
      a.S[m] = J.lv[l].msg[m];
    a.P1 = q.P1;
    a.P2 = q.P2;
    a.tau = tau;
    a.step = q.inv_depth_step;
    a.min_inv = q.min_inv_depth;
    return a;
  }

  qm::MsgPtrs adjoint(int buf) const
  {
    qm::MsgPtrs p;
    for (int m = 0; m < 4; ++m)
      p.m[m] = (float *)(adj[buf] + m * lay.dir);
    return p;
  }

  // Reverse mode over the whole pyramid, fine to coarse: the readout's
  // adjoint enters at level 0; every level recomputes its half-sweeps from
  // its starting state (all cells inherit the parents' final messages),
  // keeping each state, then runs the half-sweep adjoints backwards and hands
  // the adjoint of its starting state to the parents.
  void backward(const qm_params &q, float tau, const float *g_sparse, double *gP,
                cudaStream_t s)
  {
    const int L = q.bp_levels, D = q.num_hyp;
    const qm::KParams kp = qm::kparams(q);
    qm::check(cudaMemsetAsync(gP, 0, 2 * sizeof(double), s), "memset");
    int cur = 0;
    qm::check(cudaMemsetAsync(adj[cur], 0, 4 * lay.dir, s), "memset");
    {
      qm::DiffBp a = level_args(0, q, tau);
      const qm::MsgPtrs A = adjoint(cur);
      for (int m = 0; m < 4; ++m)
        a.A[m] = A.m[m];
      a.g_sparse = g_sparse;
      qm::launch_soft_readout(a, 1, s);
    }
    const qm::Batch B = qm::stage::single(J);
    for (int l = 0; l < L; ++l)
    {
      const int w = J.lv[l].w, h = J.lv[l].h;
      const size_t n = (size_t)w * h * D;
      const size_t slot = align256(n * sizeof(float));
      auto state = [&](int i, int m) { return (float *)(hist + ((size_t)i * 4 + m) * slot); };
      auto snapshot = [&](int i) {
        for (int m = 0; m < 4; ++m)
          qm::check(cudaMemcpyAsync(state(i, m), J.lv[l].msg[m], n * sizeof(float),
                                    cudaMemcpyDeviceToDevice, s),
                    "message snapshot");
      };
      qm::launch_msg_inherit(B, cdiv_i((long)w * h * (D / 4), qm::kFlatThreads), l, 0,
                             q.qt_max_level, s);
      snapshot(0);
      const int sweep_blocks =
          cdiv_i((long)((w + 1) / 2) * h, qm::kCellWarps * qm::bp_cells_per_warp(D));
      const int it = q.bp_iters[l];
      for (int i = 0; i < it; ++i)
      {
        qm::launch_bp_sweep_own(B, sweep_blocks, D, l, i & 1, kp, q.arith, s);
        snapshot(i + 1);
      }
      const qm::MsgPtrs A = adjoint(cur);
      for (int i = it - 1; i >= 0; --i)
      {
        qm::DiffBp a = level_args(l, q, tau);
        for (int m = 0; m < 4; ++m)
        {
          a.S[m] = state(i, m);
          a.A[m] = A.m[m];
        }
        a.parity = i & 1;
        a.gP = gP;
        qm::launch_bp_sweep_bwd(a, s);
      }
      if (l + 1 < L)
      {
        const int pw = J.lv[l + 1].w, ph = J.lv[l + 1].h;
        const qm::MsgPtrs P = adjoint(cur ^ 1);
        for (int m = 0; m < 4; ++m)
          qm::check(cudaMemsetAsync(P.m[m], 0, (size_t)pw * ph * D * sizeof(float), s),
                    "memset");
        qm::launch_msg_downsample_add(A, w, h, P, pw, ph, D, s);
        cur ^= 1;
      }
    }
    qm::check(cudaGetLastError(), "soft BP adjoint");
  }
};

// The gradient-check mode of the soft BP: the same forward and adjoint with
// every data term, message, state snapshot and adjoint in FP64 (the product
// path's BP is FP32).  Workspace: per level the FP64 data term (level 0
// widened from the FP32 cost) and four message images, the largest level's
// (iterations + 1) state snapshots, and two adjoint buffers of level 0's
// size.
struct SoftLayout64
{
  size_t lv = 0, hist = 0, dir = 0, total = 0;
};

SoftLayout64 soft_layout64(int W, int H, const qm_params &p)
{
  SoftLayout64 L;
  int w = W / 4, h = H / 4;
  L.dir = align256((size_t)w * h * p.num_hyp * sizeof(double));
  for (int l = 0; l < p.bp_levels; ++l)
  {
    const size_t n = align256((size_t)w * h * p.num_hyp * sizeof(double));
    L.lv += 5 * n;
    L.hist = std::max(L.hist, (size_t)(p.bp_iters[l] + 1) * 4 * n);
    w = (w + 1) / 2;
    h = (h + 1) / 2;
  }
  L.total = L.lv + L.hist + 2 * 4 * L.dir;
  return L;
}

struct SoftBp64
{
  int W, H, D, L;
  const uint8_t *levels;
  const float *cost;
  SoftLayout64 lay;
  int lw[qm::kMaxLevels], lh[qm::kMaxLevels];
  double *data[qm::kMaxLevels];
  qm::MsgPtrs64 msg[qm::kMaxLevels];
  char *hist = nullptr, *adj[2] = {nullptr, nullptr};

  SoftBp64(const float *cost_, int W_, int H_, const uint8_t *levels_, const qm_params &q,
           void *ws, size_t bytes)
      : W(W_), H(H_), D(q.num_hyp), L(q.bp_levels), levels(levels_), cost(cost_)
  {
    lay = soft_layout64(W, H, q);
    if (!ws || bytes < lay.total)
      throw CudaError{QM_ERR_WORKSPACE, "soft BP (FP64) workspace too small"};
    require(((uintptr_t)cost | (uintptr_t)ws) % 16 == 0,
            "cost and workspace must be 16-byte aligned");
    char *b = (char *)ws;
    size_t o = 0;
    int w = W / 4, h = H / 4;
    for (int l = 0; l < L; ++l)
    {
      const size_t n = align256((size_t)w * h * D * sizeof(double));
      lw[l] = w;
      lh[l] = h;
      data[l] = (double *)(b + o);
      o += n;
      for (int m = 0; m < 4; ++m)
      {
        msg[l].m[m] = (double *)(b + o);
        o += n;
      }
      w = (w + 1) / 2;
      h = (h + 1) / 2;
    }
    hist = b + lay.lv;
    adj[0] = hist + lay.hist;
    adj[1] = adj[0] + 4 * lay.dir;
  }

  qm::DiffBp64 level_args(int l, const qm_params &q, float tau) const
  {
    qm::DiffBp64 a;
    std::memset(&a, 0, sizeof(a));
    a.W = W;
    a.H = H;
    a.D = D;
    a.w = lw[l];
    a.h = lh[l];
    a.level = l;
    a.qt_max = q.qt_max_level;
    a.levels = levels;
    a.data = data[l];
    for (int m = 0; m < 4; ++m)
      a.S[m] = msg[l].m[m];
    a.P1 = q.P1;
    a.P2 = q.P2;
    a.tau = tau;
    a.step = q.inv_depth_step;
    a.min_inv = q.min_inv_depth;
    return a;
  }

  qm::MsgPtrs64 adjoint(int buf) const
  {
    qm::MsgPtrs64 p;
    for (int m = 0; m < 4; ++m)
      p.m[m] = (double *)(adj[buf] + m * lay.dir);
    return p;
  }

  // every cell of level l from its parent's final messages, then the
  // level's half-sweeps; snap(i) after the start and after every half-sweep
  template <class Snap>
  void sweep_level(int l, const qm_params &q, Snap &&snap, cudaStream_t s)
  {
    qm::launch_msg_inherit_all64(l + 1 < L ? &msg[l + 1] : nullptr, l + 1 < L ? lw[l + 1] : 0,
                                 msg[l], lw[l], lh[l], D, s);
    snap(0);
    for (int i = 0; i < q.bp_iters[l]; ++i)
    {
      qm::DiffBp64 a = level_args(l, q, 0.0f);
      a.parity = i & 1;
      qm::launch_bp_sweep_fwd64(a, msg[l], s);
      snap(i + 1);
    }
  }

  void forward(const qm_params &q, float tau, float *sparse, cudaStream_t s)
  {
    qm::launch_widen(cost, data[0], (long)lw[0] * lh[0] * D, s);
    for (int l = 1; l < L; ++l)
      qm::launch_pyramid64(data[l - 1], lw[l - 1], lh[l - 1], data[l], lw[l], lh[l], D, s);
    for (int l = L - 1; l >= 0; --l)
      sweep_level(l, q, [](int) {}, s);
    qm::check(cudaMemsetAsync(sparse, 0, sizeof(float) * W * H, s), "memset");
    qm::DiffBp64 a = level_args(0, q, tau);
    a.sparse = sparse;
    qm::launch_soft_readout(a, 0, s);
    qm::check(cudaGetLastError(), "soft BP (FP64)");
  }

  // as SoftBp::backward, in FP64
  void backward(const qm_params &q, float tau, const float *g_sparse, double *gP,
                cudaStream_t s)
  {
    qm::check(cudaMemsetAsync(gP, 0, 2 * sizeof(double), s), "memset");
    int cur = 0;
    qm::check(cudaMemsetAsync(adj[cur], 0, 4 * lay.dir, s), "memset");
    {
      qm::DiffBp64 a = level_args(0, q, tau);
      const qm::MsgPtrs64 A = adjoint(cur);
      for (int m = 0; m < 4; ++m)
        a.A[m] = A.m[m];
      a.g_sparse = g_sparse;
      qm::launch_soft_readout(a, 1, s);
    }
    for (int l = 0; l < L; ++l)
    {
      const size_t n = (size_t)lw[l] * lh[l] * D;
      const size_t slot = align256(n * sizeof(double));
      auto state = [&](int i, int m) { return (double *)(hist + ((size_t)i * 4 + m) * slot); };
      sweep_level(l, q,
                  [&](int i) {
                    for (int m = 0; m < 4; ++m)
                      qm::check(cudaMemcpyAsync(state(i, m), msg[l].m[m], n * sizeof(double),
                                                cudaMemcpyDeviceToDevice, s),
                                "message snapshot");
                  },
                  s);
      const qm::MsgPtrs64 A = adjoint(cur);
      for (int i = q.bp_iters[l] - 1; i >= 0; --i)
      {
        qm::DiffBp64 a = level_args(l, q, tau);
        for (int m = 0; m < 4; ++m)
        {
          a.S[m] = state(i, m);
          a.A[m] = A.m[m];
        }
        a.parity = i & 1;
        a.gP = gP;
        qm::launch_bp_sweep_bwd(a, s);
      }
      if (l + 1 < L)
      {
        const qm::MsgPtrs64 P = adjoint(cur ^ 1);
        for (int m = 0; m < 4; ++m)
          qm::check(cudaMemsetAsync(P.m[m], 0, (size_t)lw[l + 1] * lh[l + 1] * D * sizeof(double),
                                    s),
                    "memset");
        qm::launch_msg_downsample_add(A, lw[l], lh[l], P, lw[l + 1], lh[l + 1], D, s);
        cur ^= 1;
      }
    }
    qm::check(cudaGetLastError(), "soft BP (FP64) adjoint");
  }
};

qm::DiffUp upw_args(const uint8_t *img, size_t pitch, int W, int H, const qm_params *p,
                    const float *omega, void *ws, size_t bytes)
{
  check_stage_size(W, H);
  require(W % 16 == 0 && H % 8 == 0, "width must be a multiple of 16 and height of 8");
  require(img && omega && pitch >= (size_t)W, "bad argument");
  const qm_params q = params_or_default(p);
  const size_t one = align256((size_t)W * H * sizeof(double));
  if (!ws || bytes < 7 * one)
    throw CudaError{QM_ERR_WORKSPACE, "weighted upsampling workspace too small"};
  qm::DiffUp u;
  std::memset(&u, 0, sizeof(u));
  u.W = W;
  u.H = H;
  u.img = img;
  u.pitch = pitch;
  u.omega = omega;
  u.lam = q.up_lambda;
  u.sigma = q.up_sigma;
  // the reference's closing weights (depth_upsample.cu:26-37)
  u.row_closing = W % 16 != 0 ? 1.0 : 0.0;
  u.col_closing = H % 16 != 0 ? 1.0 : 0.0;
  char *b = (char *)ws;
  double **bufs[7] = {&u.sd, &u.si, &u.td, &u.ti, &u.cp, &u.ud, &u.ui};
  for (int k = 0; k < 7; ++k)
    *bufs[k] = (double *)(b + k * one);
  return u;
}

} // namespace

extern "C" {

void qm_params_default(qm_params *p)
{
  if (!p)
    return;
  std::memset(p, 0, sizeof(*p));
  p->num_hyp = 64;
  p->min_inv_depth = 0.01;
  p->inv_depth_step = (2.0 - 0.01) / 63.0;
  p->P1 = 0.003f;
  p->P2 = 0.01f;
  p->bp_levels = 4;
  p->bp_iters[0] = 4;
  p->bp_iters[1] = 10;
  p->bp_iters[2] = 10;
  p->bp_iters[3] = 10;
  p->qt_max_level = 4;
  p->qt_min_level = 2;
  p->qt_threshold = 10.0f;
  p->up_sigma = 400.0;
  p->up_lambda = 10.0;
  p->arith = QM_ARITH_REFERENCE;
}

const char *qm_last_error(void) { return qm::get_error(); }

int qm_version(void) { return 100; }

// ------------------------------------------------------------ facade

int qm_depthmap_create(qm_depthmap **out, int width, int height, float fx, float cx, float fy,
                       float cy, int semi2dense_ratio, const qm_params *params, int device)
{
  return guarded([&] {
    require(out != nullptr, "out is NULL");
    *out = nullptr;
    const qm_params p = params_or_default(params);
    qm::StreamDesc d;
    d.W = width;
    d.H = height;
    d.cam = qm::Cam{fx, fy, cx, cy};
    d.D = p.num_hyp;
    d.F = 5; // measurement slots of the reference launch (seed_matrix.cu:505)
    d.ratio = semi2dense_ratio;
    auto h = std::make_unique<qm_depthmap>();
    h->set = std::make_unique<qm::StreamSet>(device, p, std::vector<qm::StreamDesc>{d});
    h->fx = fx;
    h->fy = fy;
    h->cx = cx;
    h->cy = cy;
    h->width = width;
    h->height = height;
    *out = h.release();
  });
}

int qm_depthmap_destroy(qm_depthmap *h)
{
  return guarded([&] { delete h; });
}

int qm_depthmap_add_frame(qm_depthmap *h, const uint8_t *img, size_t stride,
                          const float T_curr_world[12], int *has_result)
{
  return guarded([&] {
    require(h && img && T_curr_world && has_result, "NULL argument");
    std::lock_guard<std::mutex> lock(h->set->mutex());
    *has_result = h->set->add_frame(0, img, stride, T_curr_world);
  });
}

int qm_depthmap_get_depth(qm_depthmap *h, float *out, size_t stride)
{
  return guarded([&] {
    require(h && out && stride >= (size_t)h->width, "bad argument");
    std::lock_guard<std::mutex> lock(h->set->mutex());
    h->set->get_depth(0, out, stride);
  });
}

int qm_depthmap_get_debug(qm_depthmap *h, float *out, size_t stride)
{
  return guarded([&] {
    require(h && out && stride >= (size_t)h->width, "bad argument");
    std::lock_guard<std::mutex> lock(h->set->mutex());
    h->set->get_debug(0, out, stride);
  });
}

int qm_depthmap_get_variance(qm_depthmap *h, float *out, size_t stride)
{
  return guarded([&] {
    require(h && out && stride >= (size_t)h->width, "bad argument");
    std::lock_guard<std::mutex> lock(h->set->mutex());
    h->set->get_variance(0, out, stride);
  });
}

int qm_depthmap_get_reference(qm_depthmap *h, uint8_t *out, size_t stride)
{
  return guarded([&] {
    require(h && out && stride >= (size_t)h->width, "bad argument");
    std::lock_guard<std::mutex> lock(h->set->mutex());
    h->set->get_reference(0, out, stride);
  });
}

int qm_depthmap_get_T_world_ref(qm_depthmap *h, float T[12])
{
  return guarded([&] {
    require(h && T, "NULL argument");
    std::lock_guard<std::mutex> lock(h->set->mutex());
    h->set->get_T_world_ref(0, T);
  });
}

int qm_depthmap_set_semidense(qm_depthmap *h, int enable)
{
  return guarded([&] {
    require(h != nullptr, "NULL handle");
    std::lock_guard<std::mutex> lock(h->set->mutex());
    h->set->set_semidense(enable != 0);
  });
}

int qm_depthmap_get_point_cloud(qm_depthmap *h, float *points, size_t capacity, int *count)
{
  return guarded([&] {
    require(h && count && (points || capacity == 0), "bad argument");
    std::lock_guard<std::mutex> lock(h->set->mutex());
    *count = h->set->get_point_cloud(0, points, capacity);
  });
}

int qm_depthmap_get_camera(qm_depthmap *h, qm_camera *cam, int *width, int *height)
{
  return guarded([&] {
    require(h != nullptr, "NULL handle");
    if (cam)
      *cam = qm_camera{h->fx, h->fy, h->cx, h->cy};
    if (width)
      *width = h->width;
    if (height)
      *height = h->height;
  });
}

// ------------------------------------------------------------- batch

int qm_batch_create(qm_batch **out, int num_streams, const qm_stream_desc *descs,
                    const qm_params *params, int device)
{
  return guarded([&] {
    require(out != nullptr, "out is NULL");
    *out = nullptr;
    require(num_streams >= 1 && descs != nullptr, "need at least one stream");
    const qm_params p = params_or_default(params);
    std::vector<qm::StreamDesc> ds;
    for (int i = 0; i < num_streams; ++i)
    {
      const qm_stream_desc &s = descs[i];
      qm::StreamDesc d;
      d.W = s.width;
      d.H = s.height;
      d.cam = qm::Cam{s.cam.fx, s.cam.fy, s.cam.cx, s.cam.cy};
      d.D = s.num_hyp > 0 ? s.num_hyp : p.num_hyp;
      d.F = s.num_slots > 0 ? s.num_slots : 5;
      d.ratio = s.semi2dense_ratio > 0 ? s.semi2dense_ratio : 1;
      ds.push_back(d);
    }
    auto b = std::make_unique<qm_batch>();
    b->set = std::make_unique<qm::StreamSet>(device, p, ds);
    *out = b.release();
  });
}

int qm_batch_destroy(qm_batch *b)
{
  return guarded([&] { delete b; });
}

int qm_batch_add_frames(qm_batch *b, const uint8_t *const *imgs, const size_t *strides,
                        const float *T_curr_world, int *has_result)
{
  return guarded([&] {
    require(b && imgs && strides && T_curr_world && has_result, "NULL argument");
    std::lock_guard<std::mutex> lock(b->set->mutex());
    b->set->add_frames(imgs, strides, T_curr_world, has_result);
  });
}

int qm_batch_submit(qm_batch *b, const uint8_t *const *imgs, const size_t *strides,
                    const float *T_curr_world, int *has_result, float *const *depth_outs,
                    const size_t *depth_strides)
{
  return guarded([&] {
    require(b && imgs && strides && T_curr_world && has_result, "NULL argument");
    std::lock_guard<std::mutex> lock(b->set->mutex());
    b->set->submit(imgs, strides, T_curr_world, has_result, depth_outs, depth_strides);
  });
}

int qm_batch_wait(qm_batch *b)
{
  return guarded([&] {
    require(b != nullptr, "NULL handle");
    std::lock_guard<std::mutex> lock(b->set->mutex());
    b->set->wait();
  });
}

int qm_batch_get_depth(qm_batch *b, int stream, float *out, size_t stride)
{
  return guarded([&] {
    require(b && out && stream >= 0 && stream < b->set->size(), "bad argument");
    require(stride >= (size_t)b->set->desc(stream).W, "stride too small");
    std::lock_guard<std::mutex> lock(b->set->mutex());
    b->set->get_depth(stream, out, stride);
  });
}

int qm_batch_get_debug(qm_batch *b, int stream, float *out, size_t stride)
{
  return guarded([&] {
    require(b && out && stream >= 0 && stream < b->set->size(), "bad argument");
    require(stride >= (size_t)b->set->desc(stream).W, "stride too small");
    std::lock_guard<std::mutex> lock(b->set->mutex());
    b->set->get_debug(stream, out, stride);
  });
}

int qm_batch_run_resident(qm_batch *b)
{
  return guarded([&] {
    require(b != nullptr, "NULL handle");
    std::lock_guard<std::mutex> lock(b->set->mutex());
    b->set->run_resident();
  });
}

int qm_batch_get_variance(qm_batch *b, int stream, float *out, size_t stride)
{
  return guarded([&] {
    require(b && out && stream >= 0 && stream < b->set->size() &&
                stride >= (size_t)b->set->desc(stream).W,
            "bad argument");
    std::lock_guard<std::mutex> lock(b->set->mutex());
    b->set->get_variance(stream, out, stride);
  });
}

int qm_batch_get_point_cloud(qm_batch *b, int stream, float *points, size_t capacity,
                             int *count)
{
  return guarded([&] {
    require(b && count && (points || capacity == 0) && stream >= 0 && stream < b->set->size(),
            "bad argument");
    std::lock_guard<std::mutex> lock(b->set->mutex());
    *count = b->set->get_point_cloud(stream, points, capacity);
  });
}

int qm_batch_device_depth(qm_batch *b, int stream, const float **dev_ptr)
{
  return guarded([&] {
    require(b && dev_ptr && stream >= 0 && stream < b->set->size(), "bad argument");
    std::lock_guard<std::mutex> lock(b->set->mutex());
    b->set->wait();
    *dev_ptr = b->set->device_depth(stream);
  });
}

int qm_batch_set_branches(qm_batch *b, int branches)
{
  return guarded([&] {
    require(b != nullptr && branches >= 1 && branches <= 4, "bad argument");
    std::lock_guard<std::mutex> lock(b->set->mutex());
    b->set->wait();
    b->set->engine().set_branches(branches);
  });
}

int qm_batch_set_semidense(qm_batch *b, int enable)
{
  return guarded([&] {
    require(b != nullptr, "NULL handle");
    std::lock_guard<std::mutex> lock(b->set->mutex());
    b->set->set_semidense(enable != 0);
  });
}

int qm_batch_set_graphs(qm_batch *b, int enable)
{
  return guarded([&] {
    require(b != nullptr, "NULL handle");
    b->set->engine().set_graphs(enable != 0);
  });
}

int qm_batch_get_depths(qm_batch *b, int n, const int *streams, float *const *outs,
                        const size_t *strides)
{
  return guarded([&] {
    require(b && n >= 0 && (n == 0 || (streams && outs && strides)), "bad argument");
    std::lock_guard<std::mutex> lock(b->set->mutex());
    b->set->get_depths(streams, n, outs, strides);
  });
}

int qm_batch_set_group_bytes(qm_batch *b, size_t bytes)
{
  return guarded([&] {
    require(b != nullptr, "NULL handle");
    b->set->engine().set_group_bytes(bytes);
  });
}

int qm_batch_set_coarse_bp(qm_batch *b, int max_cells)
{
  return guarded([&] {
    require(b != nullptr, "NULL handle");
    require(max_cells >= 0, "max_cells must be >= 0");
    std::lock_guard<std::mutex> lock(b->set->mutex());
    b->set->engine().set_coarse_cells(max_cells);
  });
}

int qm_batch_set_stagger(qm_batch *b, int enable)
{
  return guarded([&] {
    require(b != nullptr, "NULL handle");
    std::lock_guard<std::mutex> lock(b->set->mutex());
    b->set->engine().set_stagger(enable != 0);
  });
}

int qm_batch_set_autotune(qm_batch *b, int enable)
{
  return guarded([&] {
    require(b != nullptr, "NULL handle");
    std::lock_guard<std::mutex> lock(b->set->mutex());
    b->set->wait();
    b->set->engine().set_autotune(enable != 0);
  });
}

int qm_batch_set_tune(qm_batch *b, const qm_tune *t)
{
  return guarded([&] {
    require(b && t, "NULL argument");
    std::lock_guard<std::mutex> lock(b->set->mutex());
    b->set->wait();
    qm::Tune u;
    u.sweep_warps = t->sweep_warps;
    u.extract_warps = t->extract_warps;
    u.row_warps = t->row_warps;
    u.col_lines = t->col_lines;
    // 0 (a qm_tune initialised with the four block shapes only): the default
    u.cost_blocks = t->cost_blocks == 0 ? qm::kCostBlocks : t->cost_blocks;
    b->set->engine().set_tune(u);
  });
}

int qm_batch_get_tune(qm_batch *b, qm_tune *t)
{
  return guarded([&] {
    require(b && t, "NULL argument");
    const qm::Tune u = b->set->engine().last_tune();
    t->sweep_warps = u.sweep_warps;
    t->extract_warps = u.extract_warps;
    t->row_warps = u.row_warps;
    t->col_lines = u.col_lines;
    t->cost_blocks = u.cost_blocks;
  });
}

int qm_batch_last_launches(qm_batch *b, int *count)
{
  return guarded([&] {
    require(b && count, "NULL argument");
    *count = b->set->engine().last_launches();
  });
}

int qm_batch_stream(qm_batch *b, void **stream)
{
  return guarded([&] {
    require(b && stream, "NULL argument");
    *stream = reinterpret_cast<void *>(b->set->engine().stream());
  });
}

int qm_batch_profile(qm_batch *b, float ms[QM_NUM_KERNEL_KINDS],
                     int launches[QM_NUM_KERNEL_KINDS])
{
  static_assert(QM_NUM_KERNEL_KINDS == qm::kNumKinds, "kernel kind count");
  return guarded([&] {
    require(b && ms && launches, "NULL argument");
    std::lock_guard<std::mutex> lock(b->set->mutex());
    b->set->profile_resident(ms, launches);
  });
}

// ------------------------------------------------------------ stages

int qm_quadtree(const uint8_t *img, size_t img_pitch, int width, int height, const qm_params *p,
                uint8_t *levels, void *stream)
{
  return guarded([&] {
    check_stage_size(width, height);
    require(img && levels && img_pitch >= (size_t)width, "bad argument");
    const qm_params q = params_or_default(p);
    qm::JobDesc J = base_desc(width, height, q);
    J.ref = img;
    J.ref_pitch = (int)img_pitch;
    J.levels = levels;
    run_stage(J, q, stage_shape(width, height, q, 1, nullptr), "quadtree", stream);
  });
}

int qm_cost_volume(const uint8_t *ref, size_t ref_pitch, int width, int height,
                   const qm_camera *cam, const uint8_t *levels, int num_slots,
                   const uint8_t *const *slots, size_t slot_pitch, const float *T_slot_ref,
                   const qm_params *p, float *cost, void *stream)
{
  return guarded([&] {
    check_stage_size(width, height);
    require(ref && cam && levels && slots && T_slot_ref && cost, "NULL argument");
    require(ref_pitch >= (size_t)width && slot_pitch >= (size_t)width, "pitch too small");
    require(num_slots >= 1 && num_slots <= QM_MAX_SLOTS, "num_slots must be in [1, 32]");
    const qm_params q = params_or_default(p);
    qm::JobDesc J = base_desc(width, height, q);
    J.F = num_slots;
    J.fx = cam->fx;
    J.fy = cam->fy;
    J.cx = cam->cx;
    J.cy = cam->cy;
    J.ref = ref;
    J.ref_pitch = (int)ref_pitch;
    J.slot_pitch = (int)slot_pitch;
    J.levels = const_cast<uint8_t *>(levels);
    J.lv[0].data = cost;
    qm::SlotInline si;
    std::memset(&si, 0, sizeof(si));
    for (int f = 0; f < num_slots; ++f)
      require(slots[f] != nullptr, "NULL slot image");
    J.F = qm::dedupe_slots(num_slots, slots, T_slot_ref, si.ptr, si.T, si.w);
    run_stage(J, q, stage_shape(width, height, q, num_slots, cam), "cost", stream, &si);
  });
}

int qm_bp_workspace_size(int width, int height, const qm_params *p, size_t *bytes)
{
  return guarded([&] {
    check_stage_size(width, height);
    require(bytes != nullptr, "NULL argument");
    const qm_params q = params_or_default(p);
    *bytes = bp_workspace(width, height, q);
  });
}

int qm_bp_extract(const float *cost, int width, int height, const uint8_t *levels,
                  const qm_params *p, float *sparse, int32_t *labels, float *messages,
                  void *workspace, size_t workspace_bytes, void *stream)
{
  return guarded([&] {
    check_stage_size(width, height);
    require(cost && levels && sparse, "NULL argument");
    const qm_params q = params_or_default(p);
    const size_t need = bp_workspace(width, height, q);
    if (workspace_bytes < need || !workspace)
      throw CudaError{QM_ERR_WORKSPACE, "BP workspace too small"};
    // the pyramid and message kernels move float4 groups
    require(((uintptr_t)cost | (uintptr_t)messages | (uintptr_t)workspace) % 16 == 0,
            "cost, messages and workspace must be 16-byte aligned");
    qm::JobDesc J = base_desc(width, height, q);
    J.levels = const_cast<uint8_t *>(levels);
    J.sparse = sparse;
    J.labels = labels;
    char *ws = (char *)workspace;
    size_t o = 0;
    int w = width / 4, h = height / 4;
    for (int l = 0; l < q.bp_levels; ++l)
    {
      const size_t n = (size_t)w * h * q.num_hyp * sizeof(float);
      J.lv[l].w = w;
      J.lv[l].h = h;
      if (l == 0)
        J.lv[l].data = const_cast<float *>(cost);
      else
      {
        J.lv[l].data = (float *)(ws + o);
        o += align256(n);
      }
      for (int m = 0; m < 4; ++m)
      {
        J.lv[l].msg[m] = (float *)(ws + o);
        o += align256(n);
        if (l == 0 && messages)
          J.lv[l].msg[m] = messages + (size_t)m * w * h * q.num_hyp;
      }
      w = (w + 1) / 2;
      h = (h + 1) / 2;
    }
    run_stage(J, q, stage_shape(width, height, q, 1, nullptr), "bp", stream);
  });
}

int qm_upsample_workspace_size(int width, int height, size_t *bytes)
{
  return guarded([&] {
    check_stage_size(width, height);
    require(bytes != nullptr, "NULL argument");
    *bytes = upsample_workspace(width, height);
  });
}

int qm_upsample(const float *sparse, const uint8_t *img, size_t img_pitch, int width, int height,
                const qm_params *p, float *dense, void *workspace, size_t workspace_bytes,
                void *stream)
{
  return guarded([&] {
    check_stage_size(width, height);
    require(width % 16 == 0 && height % 8 == 0,
            "width must be a multiple of 16 and height of 8");
    require(width <= qm::kMaxRowLen && height <= qm::kMaxColLen,
            "upsampling supports at most 4096 x 2048");
    require(sparse && img && dense && img_pitch >= (size_t)width, "bad argument");
    const qm_params q = params_or_default(p);
    if (workspace_bytes < upsample_workspace(width, height) || !workspace)
      throw CudaError{QM_ERR_WORKSPACE, "upsample workspace too small"};
    qm::JobDesc J = base_desc(width, height, q);
    J.ref = img;
    J.ref_pitch = (int)img_pitch;
    J.sparse = const_cast<float *>(sparse);
    J.dense = dense;
    J.rowres = (float2 *)workspace;
    run_stage(J, q, stage_shape(width, height, q, 1, nullptr), "upsample", stream);
  });
}

int qm_fuse_workspace_size(int width, int height, size_t *bytes)
{
  return guarded([&] {
    check_stage_size(width, height);
    require(bytes != nullptr, "NULL argument");
    *bytes = fuse_workspace(width, height);
  });
}

int qm_fuse(float *depth, float *seeds_in, float *seeds_out, const float T_income_last[12],
            const qm_camera *cam, int width, int height, const qm_params *p, int32_t *table,
            void *workspace, size_t workspace_bytes, void *stream)
{
  return guarded([&] {
    check_stage_size(width, height);
    require(depth && seeds_in && seeds_out && T_income_last && cam && table, "NULL argument");
    const qm_params q = params_or_default(p);
    if (workspace_bytes < fuse_workspace(width, height) || !workspace)
      throw CudaError{QM_ERR_WORKSPACE, "fuse workspace too small"};
    qm::JobDesc J = base_desc(width, height, q);
    J.fx = cam->fx;
    J.fy = cam->fy;
    J.cx = cam->cx;
    J.cy = cam->cy;
    J.dense = depth;
    J.seeds_in = reinterpret_cast<float4 *>(seeds_in);
    J.seeds_out = reinterpret_cast<float4 *>(seeds_out);
    J.table = table;
    J.zkey = (unsigned long long *)workspace;
    std::memcpy(J.Tf, T_income_last, 12 * sizeof(float));
    qm::check(cudaMemsetAsync(workspace, 0xff, fuse_workspace(width, height), as_stream(stream)),
              "workspace reset");
    run_stage(J, q, stage_shape(width, height, q, 1, cam), "fuse", stream);
  });
}

int qm_point_cloud_workspace_size(int width, int height, size_t *bytes)
{
  return guarded([&] {
    check_stage_size(width, height);
    require(bytes != nullptr, "NULL argument");
    *bytes = qm::point_cloud_workspace(width, height);
  });
}

int qm_point_cloud(const float *depth, size_t depth_stride, const uint8_t *ref, size_t ref_pitch,
                   int width, int height, const qm_camera *cam, const float T_world_ref[12],
                   float *points, int *count, void *workspace, size_t workspace_bytes,
                   void *stream)
{
  return guarded([&] {
    check_stage_size(width, height);
    require(depth && ref && cam && T_world_ref && points && count, "NULL argument");
    require(depth_stride >= (size_t)width && ref_pitch >= (size_t)width, "bad stride");
    if (workspace_bytes < qm::point_cloud_workspace(width, height) || !workspace)
      throw CudaError{QM_ERR_WORKSPACE, "point-cloud workspace too small"};
    qm::Cam c{cam->fx, cam->fy, cam->cx, cam->cy};
    qm::launch_point_cloud(depth, depth_stride, ref, ref_pitch, width, height, c, T_world_ref,
                           reinterpret_cast<float4 *>(points), count, workspace,
                           as_stream(stream));
    qm::check(cudaGetLastError(), "point cloud");
  });
}

// ------------------------------------------------------ semi-dense tracker

namespace
{

struct SdLayout
{
  size_t pitch, key_f, inc_f, trk2, dep2, zkey, total;
};

SdLayout sd_layout(int W, int H)
{
  auto a512 = [](size_t x) { return (x + 511) & ~size_t(511); };
  SdLayout L;
  L.pitch = qm::sd_texture_pitch(W);
  const size_t img = a512(L.pitch * H * sizeof(float));
  const size_t P = (size_t)W * H;
  L.key_f = 0;
  L.inc_f = L.key_f + img;
  L.trk2 = L.inc_f + img;
  L.dep2 = L.trk2 + a512(P * sizeof(float4));
  L.zkey = L.dep2 + a512(P * sizeof(float4));
  L.total = L.zkey + a512(P * sizeof(unsigned long long));
  return L;
}

} // namespace

int qm_semidense_workspace_size(int width, int height, size_t *bytes)
{
  return guarded([&] {
    check_stage_size(width, height);
    require(bytes != nullptr, "NULL argument");
    *bytes = sd_layout(width, height).total;
  });
}

int qm_semidense_step(const uint8_t *key, const uint8_t *inc, int width, int height,
                      const qm_camera *cam, const float T_income_key[12], int mode, int arith,
                      float *trk, float *dep, float *debug, void *workspace,
                      size_t workspace_bytes, void *stream)
{
  return guarded([&] {
    check_stage_size(width, height);
    require(inc && cam && T_income_key && trk && dep && debug, "NULL argument");
    require(mode == QM_SD_INIT || mode == QM_SD_UPDATE || mode == QM_SD_SWITCH, "bad mode");
    require(mode == QM_SD_INIT || key != nullptr, "keyframe image missing");
    require(arith == QM_ARITH_REFERENCE || arith == QM_ARITH_IEEE, "bad arith");
    const SdLayout L = sd_layout(width, height);
    if (!workspace || workspace_bytes < L.total)
      throw CudaError{QM_ERR_WORKSPACE, "semi-dense workspace too small"};
    const cudaStream_t s = as_stream(stream);
    char *ws = static_cast<char *>(workspace);
    qm::SdBatch B;
    std::memset(&B, 0, sizeof(B));
    qm::SdJob &J = B.one;
    J.W = width;
    J.H = height;
    J.fx = cam->fx;
    J.fy = cam->fy;
    J.cx = cam->cx;
    J.cy = cam->cy;
    J.mode = mode;
    J.inc = inc;
    J.inc_f = reinterpret_cast<float *>(ws + L.inc_f);
    J.key_f = reinterpret_cast<float *>(ws + L.key_f);
    J.pitch = L.pitch;
    J.trk[0] = reinterpret_cast<float4 *>(trk);
    J.dep[0] = reinterpret_cast<float4 *>(dep);
    J.trk[1] = reinterpret_cast<float4 *>(ws + L.trk2);
    J.dep[1] = reinterpret_cast<float4 *>(ws + L.dep2);
    J.cur = 0;
    J.debug = debug;
    J.zkey = reinterpret_cast<unsigned long long *>(ws + L.zkey);
    std::memcpy(J.T, T_income_key, 12 * sizeof(float));
    qm::check(cudaMemsetAsync(J.zkey, 0xff, (size_t)width * height * sizeof(unsigned long long), s),
              "workspace reset");
    if (key)
      qm::launch_u8_to_f32(key, width, height, const_cast<float *>(J.key_f), L.pitch, s);
    const bool ref = arith == QM_ARITH_REFERENCE;
    if (ref)
    {
      J.key_tex = qm::sd_make_texture(J.key_f, width, height, L.pitch);
      J.inc_tex = qm::sd_make_texture(J.inc_f, width, height, L.pitch);
      if (!J.key_tex || !J.inc_tex)
      {
        if (J.key_tex)
          cudaDestroyTextureObject(J.key_tex);
        if (J.inc_tex)
          cudaDestroyTextureObject(J.inc_tex);
        throw CudaError{QM_ERR_CUDA, "texture object creation failed"};
      }
    }
    qm::launch_semidense(B, qm::sd_blocks(width, height), ref ? 0 : 1, s);
    const cudaError_t e = cudaGetLastError();
    if (ref)
    {
      const cudaError_t w = cudaStreamSynchronize(s);
      cudaDestroyTextureObject(J.key_tex);
      cudaDestroyTextureObject(J.inc_tex);
      qm::check(w, "semi-dense step");
    }
    qm::check(e, "semi-dense step");
  });
}

// ------------------------------------------------------ differentiable path

int qm_bp_soft_workspace_size(int width, int height, const qm_params *p, size_t *bytes)
{
  return guarded([&] {
    check_stage_size(width, height);
    require(bytes != nullptr, "NULL argument");
    *bytes = soft_layout(width, height, params_or_default(p)).total;
  });
}

int qm_bp_soft_forward(const float *cost, int width, int height, const uint8_t *levels,
                       const qm_params *p, float tau, float *sparse, void *workspace,
                       size_t workspace_bytes, void *stream)
{
  return guarded([&] {
    check_stage_size(width, height);
    require(cost && levels && sparse && tau > 0.0f, "NULL argument or tau <= 0");
    const qm_params q = params_or_default(p);
    SoftBp sb(cost, width, height, levels, q, workspace, workspace_bytes);
    const cudaStream_t s = as_stream(stream);
    qm::check(cudaMemsetAsync(sparse, 0, sizeof(float) * width * height, s), "memset");
    sb.J.sparse = sparse;
    // hierarchical BP (its hard extraction is overwritten by the soft readout)
    run_stage(sb.J, q, stage_shape(width, height, q, 1, nullptr), "bp", stream);
    qm::DiffBp a = sb.level_args(0, q, tau);
    a.sparse = sparse;
    qm::launch_soft_readout(a, 0, s);
    qm::check(cudaGetLastError(), "soft readout");
  });
}

int qm_bp_soft_backward(const float *cost, int width, int height, const uint8_t *levels,
                        const qm_params *p, float tau, const float *grad_sparse,
                        double *grad_penalties, void *workspace, size_t workspace_bytes,
                        void *stream)
{
  return guarded([&] {
    check_stage_size(width, height);
    require(cost && levels && grad_sparse && grad_penalties && tau > 0.0f,
            "NULL argument or tau <= 0");
    const qm_params q = params_or_default(p);
    SoftBp sb(cost, width, height, levels, q, workspace, workspace_bytes);
    sb.backward(q, tau, grad_sparse, grad_penalties, as_stream(stream));
  });
}

int qm_bp_soft64_workspace_size(int width, int height, const qm_params *p, size_t *bytes)
{
  return guarded([&] {
    check_stage_size(width, height);
    require(bytes != nullptr, "NULL argument");
    *bytes = soft_layout64(width, height, params_or_default(p)).total;
  });
}

int qm_bp_soft64_forward(const float *cost, int width, int height, const uint8_t *levels,
                         const qm_params *p, float tau, float *sparse, void *workspace,
                         size_t workspace_bytes, void *stream)
{
  return guarded([&] {
    check_stage_size(width, height);
    require(cost && levels && sparse && tau > 0.0f, "NULL argument or tau <= 0");
    const qm_params q = params_or_default(p);
    SoftBp64 sb(cost, width, height, levels, q, workspace, workspace_bytes);
    sb.forward(q, tau, sparse, as_stream(stream));
  });
}

int qm_bp_soft64_backward(const float *cost, int width, int height, const uint8_t *levels,
                          const qm_params *p, float tau, const float *grad_sparse,
                          double *grad_penalties, void *workspace, size_t workspace_bytes,
                          void *stream)
{
  return guarded([&] {
    check_stage_size(width, height);
    require(cost && levels && grad_sparse && grad_penalties && tau > 0.0f,
            "NULL argument or tau <= 0");
    const qm_params q = params_or_default(p);
    SoftBp64 sb(cost, width, height, levels, q, workspace, workspace_bytes);
    sb.backward(q, tau, grad_sparse, grad_penalties, as_stream(stream));
  });
}

int qm_upsample_w_workspace_size(int width, int height, size_t *bytes)
{
  return guarded([&] {
    check_stage_size(width, height);
    require(bytes != nullptr, "NULL argument");
    *bytes = align256((size_t)width * height * sizeof(double)) * 7;
  });
}

int qm_upsample_w_forward(const float *sparse, const uint8_t *img, size_t img_pitch, int width,
                          int height, const qm_params *p, const float *omega, float *dense,
                          void *workspace, size_t workspace_bytes, void *stream)
{
  return guarded([&] {
    qm::DiffUp u = upw_args(img, img_pitch, width, height, p, omega, workspace, workspace_bytes);
    require(sparse && dense, "NULL argument");
    u.sparse = sparse;
    u.dense = dense;
    qm::launch_upw_forward(u, as_stream(stream));
    qm::check(cudaGetLastError(), "weighted upsampling");
  });
}

int qm_upsample_w_backward(const uint8_t *img, size_t img_pitch, int width, int height,
                           const qm_params *p, const float *omega, const float *grad_dense,
                           float *grad_sparse, float *grad_omega, void *workspace,
                           size_t workspace_bytes, void *stream)
{
  return guarded([&] {
    qm::DiffUp u = upw_args(img, img_pitch, width, height, p, omega, workspace, workspace_bytes);
    require(grad_dense && grad_sparse && grad_omega, "NULL argument");
    u.g_dense = grad_dense;
    u.g_sparse = grad_sparse;
    u.g_omega = grad_omega;
    qm::launch_upw_backward(u, as_stream(stream));
    qm::check(cudaGetLastError(), "weighted upsampling adjoint");
  });
}

int qm_fuse_backward(const float *depth_in, const float *seeds_in, const int32_t *table,
                     int width, int height, const float *grad_fused, float *grad_depth,
                     void *stream)
{
  return guarded([&] {
    check_stage_size(width, height);
    require(depth_in && seeds_in && table && grad_fused && grad_depth, "NULL argument");
    qm::DiffFuse f;
    f.W = width;
    f.H = height;
    f.depth_in = depth_in;
    f.seeds_in = reinterpret_cast<const float4 *>(seeds_in);
    f.table = table;
    f.g_fused = grad_fused;
    f.g_depth = grad_depth;
    qm::launch_fuse_bwd(f, as_stream(stream));
    qm::check(cudaGetLastError(), "fusion adjoint");
  });
}

} // extern "C"
