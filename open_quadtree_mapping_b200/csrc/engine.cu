// Host engine of the dense pipeline (see engine.h).
//
// Stage order of one run, after SeedMatrix::extract_depth and
// fuse_output_depth (seed_matrix.cu:448-597):
//   quadtree -> cost -> pyramid(1..L-1) ->
//   for level L-1..0: bp half-sweeps (the first two also write the
//     inherited messages; a separate inheritance pass only at levels with
//     fewer than two) (+ extraction at level 0) ->
//   row solve (also resets the fusion keys) -> column solve ->
//   fuse transform -> fuse update (hole filling inside).
// Every stage is one launch over all active jobs (one per hypothesis count
// for the warp-per-cell BP kernels); optionally the BP stages of a level run
// over consecutive job ranges whose level working set fits a byte budget, so
// the half-sweeps of a range re-read their costs and messages from L2.  The
// reference runs 60-70 launches per keyframe with a cudaDeviceSynchronize
// after most and ~25 device allocations; here a batch needs no allocation,
// and the whole sequence is captured once per active set and replayed as a
// graph.
#include "engine.h"

#include <algorithm>
#include <cstring>
#include <cmath>
#include <set>

namespace qm
{

namespace
{
thread_local std::string t_err;

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

int cdiv(long a, long b) { return (int)((a + b - 1) / b); }

// Stage indices for L pyramid levels.
struct Stages
{
  int L;
  int qt() const { return 0; }
  int cost() const { return 1; }
  int pyr(int l) const { return 2 + (l - 1); } // l = 1..L-1
  int inherit(int l) const { return 1 + L + l; } // l = 0..L-1
  int sweep(int l) const { return 1 + 2 * L + l; }
  int extract() const { return 1 + 3 * L; }
  int row() const { return 2 + 3 * L; }
  int col() const { return 3 + 3 * L; }
  int ftrans() const { return 4 + 3 * L; }
  int fupd() const { return 5 + 3 * L; } // hole filling + posterior update
  int count() const { return 6 + 3 * L; }
};

std::vector<int> stage_blocks(const Shape &s, const JobLayout &lay, const qm_params &p,
                              const Tune &tune)
{
  const Stages st{p.bp_levels};
  std::vector<int> b(st.count(), 0);
  const int L = p.bp_levels;
  const int D = s.D;
  b[st.qt()] = quadtree_blocks(s.W, s.H, p.qt_max_level);
  b[st.cost()] = cost_blocks(lay.lw[0], lay.lh[0]);
  // pyramid and message kernels move float4 groups of hypotheses
  for (int l = 1; l < L; ++l)
    b[st.pyr(l)] = cdiv((long)lay.lw[l] * lay.lh[l] * (D / 4), kFlatThreads);
  for (int l = 0; l < L; ++l)
    b[st.inherit(l)] = cdiv((long)lay.lw[l] * lay.lh[l] * (D / 4), kFlatThreads);
  // BP cells per block of the half-sweeps and of the extraction
  const int spb = tune.sweep_warps * bp_cells_per_warp(D);
  const int epb = tune.extract_warps * bp_cells_per_warp(D);
  for (int l = 0; l < L; ++l)
    b[st.sweep(l)] = cdiv((long)((lay.lw[l] + 1) / 2) * lay.lh[l], spb);
  b[st.extract()] = cdiv((long)lay.lw[0] * lay.lh[0], epb);
  b[st.row()] = cdiv(s.H, tune.row_warps);
  b[st.col()] = cdiv(s.W, tune.col_lines);
  b[st.ftrans()] = cdiv((long)s.W * s.H, kFlatThreads * kFuseTransformPx);
  b[st.fupd()] = cdiv((long)s.W * s.H, kFlatThreads * kFuseUpdatePx);
  return b;
}

// Block layout of every stage over the jobs of one launch sequence.
struct StageTable
{
  int n = 0;                       // jobs
  std::vector<int> hprefix;        // host, stage s: [s*(n+1), (s+1)*(n+1))
  std::vector<const int *> prefix; // device copy per stage (null: one inline job)
  std::vector<int> uniform;        // per stage: blocks per job when all agree, else 0
  std::vector<int> dvals;          // hypothesis counts present
  std::vector<size_t> level_bytes; // per job and BP level: data + messages
  std::vector<long> level_cells;   // per BP level: largest cell count over the jobs
  int max_w = 0, max_h = 0;        // longest lines of the row / column solves
  Tune tune;                       // launch shapes the blocks were counted for

  int begin(int stage, int j) const { return hprefix[(size_t)stage * (n + 1) + j]; }
  int blocks(int stage) const { return begin(stage, n); }

  void add_jobs(const std::vector<std::vector<int>> &per_job, const std::vector<int> &ds)
  {
    n = (int)per_job.size();
    const int ns = n ? (int)per_job[0].size() : 0;
    hprefix.assign((size_t)ns * (n + 1), 0);
    uniform.assign(ns, 0);
    for (int st = 0; st < ns; ++st)
    {
      bool same = true;
      for (int j = 0; j < n; ++j)
      {
        hprefix[(size_t)st * (n + 1) + j + 1] = hprefix[(size_t)st * (n + 1) + j] + per_job[j][st];
        same = same && per_job[j][st] == per_job[0][st];
      }
      uniform[st] = (same && n > 0) ? per_job[0][st] : 0;
    }
    std::set<int> u(ds.begin(), ds.end());
    dvals.assign(u.begin(), u.end());
  }
};

// Consecutive job ranges [g[i], g[i+1]) whose BP level-`level` working sets
// stay within `budget` bytes (at least one job per range); budget 0 = one
// range.  Running the sweeps of a level range by range keeps that range's
// costs and messages resident in L2 across the half-sweeps.
std::vector<int> job_groups(const StageTable &T, int level, int L, size_t budget, int ja, int jb)
{
  std::vector<int> g{ja};
  size_t acc = 0;
  for (int j = ja; j < jb; ++j)
  {
    const size_t b = T.level_bytes.empty() ? 0 : T.level_bytes[(size_t)j * L + level];
    if (budget > 0 && j > g.back() && acc + b > budget)
    {
      g.push_back(j);
      acc = 0;
    }
    acc += b;
  }
  g.push_back(jb);
  return g;
}

// Launches stages [first, last] of the sequence for jobs [ja, jb) (jb < 0:
// all).  When `prof` is given, every launch is bracketed by a pair of events
// recorded on `s`.  Returns the number of kernel launches.
int enqueue_range(const Batch &B, const StageTable &T, const qm_params &p, size_t group_bytes,
                  int coarse_cells, int first, int last, cudaStream_t s,
                  LaunchProfile *prof = nullptr, int ja = 0, int jb = -1)
{
  if (jb < 0)
    jb = T.n;
  const Stages st{p.bp_levels};
  const int L = p.bp_levels;
  const KParams kp = kparams(p);
  const int ar = p.arith;
  int n = 0;
  auto in = [&](int stage) { return stage >= first && stage <= last && T.blocks(stage) > 0; };
  // the batch of stage `stage` restricted to jobs [j0, j1), and its grid
  auto at = [&](int stage, int j0, int j1, int &grid) {
    Batch b = B;
    b.prefix = T.prefix.empty() ? nullptr : T.prefix[stage];
    b.uniform = T.uniform[stage];
    b.block0 = T.begin(stage, j0);
    grid = T.begin(stage, j1) - b.block0;
    return b;
  };
  auto launch = [&](int kind, auto &&fn) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (prof)
    {
      check(cudaEventCreate(&e0), "event");
      check(cudaEventCreate(&e1), "event");
      check(cudaEventRecord(e0, s), "event");
    }
    fn();
    if (prof)
    {
      check(cudaEventRecord(e1, s), "event");
      prof->marks.push_back({kind, e0, e1});
    }
    ++n;
  };
  // one launch of `stage` over all jobs
  auto all = [&](int kind, int stage, auto &&fn) {
    if (!in(stage))
      return;
    int grid = 0;
    const Batch b = at(stage, ja, jb, grid);
    if (grid > 0)
      launch(kind, [&] { fn(b, grid); });
  };
  all(kQuadtree, st.qt(), [&](const Batch &b, int g) { launch_quadtree(b, g, kp, s); });
  const int max_d = T.dvals.empty() ? 0 : T.dvals.back();
  all(kCost, st.cost(),
      [&](const Batch &b, int g) { launch_cost(b, g, ar, max_d, s, T.tune.cost_blocks); });
  for (int l = 1; l < L; ++l)
    all(kPyramid, st.pyr(l), [&](const Batch &b, int g) { launch_pyramid(b, g, l, s); });
  // BP, coarse to fine.  The top levels lc..L-1 whose cells are few (and
  // which have two or more half-sweeps) run as one cluster launch per
  // hypothesis count; below them each level runs job range by job range
  // (message inheritance, half-sweeps, and at level 0 the extraction)
  int lc = L;
  if (coarse_cells > 0 && (int)T.level_cells.size() == L)
    while (lc > 0 && p.bp_iters[lc - 1] >= 2 && T.level_cells[lc - 1] <= coarse_cells &&
           in(st.sweep(lc - 1)))
      --lc;
  if (lc < L && jb > ja)
  {
    CoarsePlan cp;
    std::memset(&cp, 0, sizeof(cp));
    cp.lo = lc;
    cp.hi = L - 1;
    for (int l = 0; l < L; ++l)
      cp.iters[l] = p.bp_iters[l];
    for (int d : T.dvals)
      launch(kSweep, [&] { launch_bp_coarse(B, ja, jb - ja, d, cp, kp, ar, s); });
  }
  for (int l = L - 1; l >= 0; --l)
  {
    const std::vector<int> groups = job_groups(T, l, L, group_bytes, ja, jb);
    for (size_t gi = 0; gi + 1 < groups.size(); ++gi)
    {
      const int j0 = groups[gi], j1 = groups[gi + 1];
      int grid = 0;
      // with two or more half-sweeps the first two write the inherited
      // messages themselves (no separate pass)
      const bool fold = p.bp_iters[l] >= 2;
      if (l >= lc)
        ; // swept by the coarse launch
      else if (!fold && in(st.inherit(l)))
      {
        const Batch b = at(st.inherit(l), j0, j1, grid);
        if (grid > 0)
          launch(kMsgInit, [&] {
            launch_msg_inherit(b, grid, l, p.bp_iters[l], p.qt_max_level, s);
          });
      }
      if (l < lc && in(st.sweep(l)))
      {
        // consecutive half-sweeps walk the cells in opposite orders, so each
        // starts on the messages its predecessor wrote last (still in L2)
        Batch b = at(st.sweep(l), j0, j1, grid);
        if (grid > 0)
          for (int it = 0; it < p.bp_iters[l]; ++it)
          {
            b.rev = it & 1;
            for (int d : T.dvals)
              launch(kSweep, [&] {
                launch_bp_sweep(b, grid, d, l, it, kp, ar, s, T.tune.sweep_warps,
                                fold && in(st.inherit(l)) ? 1 : 0);
              });
          }
      }
      if (l == 0 && in(st.extract()))
      {
        // against the order of the level's last half-sweep (see above)
        Batch b = at(st.extract(), j0, j1, grid);
        b.rev = (l < lc && p.bp_iters[0] > 0) ? 1 - ((p.bp_iters[0] - 1) & 1) : 0;
        if (grid > 0)
          for (int d : T.dvals)
            launch(kExtract, [&] { launch_extract(b, grid, d, ar, s, T.tune.extract_warps); });
      }
    }
  }
  all(kRowSolve, st.row(), [&](const Batch &b, int g) {
    launch_row_solve(b, g, kp, ar, T.max_w, s, T.tune.row_warps);
  });
  all(kColSolve, st.col(), [&](const Batch &b, int g) {
    launch_col_solve(b, g, kp, ar, T.max_h, s, T.tune.col_lines);
  });
  all(kFuseTransform, st.ftrans(),
      [&](const Batch &b, int g) { launch_fuse_transform(b, g, ar, s); });
  all(kFuseUpdate, st.fupd(), [&](const Batch &b, int g) { launch_fuse_update(b, g, s); });
  check(cudaGetLastError(), "kernel launch");
  return n;
}

} // namespace

void set_error(const std::string &msg) { t_err = msg; }
const char *get_error() { return t_err.c_str(); }

void check(cudaError_t e, const char *what)
{
  if (e != cudaSuccess)
  {
    cudaGetLastError(); // clear a sticky launch error of this call
    throw CudaError{e == cudaErrorMemoryAllocation ? QM_ERR_NO_MEMORY : QM_ERR_CUDA,
                    std::string(what) + ": " + cudaGetErrorString(e)};
  }
}

KParams kparams(const qm_params &p)
{
  KParams k;
  k.P1 = p.P1;
  k.P2 = p.P2;
  k.qt_max = p.qt_max_level;
  k.qt_min = p.qt_min_level;
  k.qt_thr = p.qt_threshold;
  k.up_sigma = p.up_sigma;
  k.up_lambda = p.up_lambda;
  return k;
}

bool rigid_enough(const float *T)
{
  for (int k = 0; k < 12; ++k)
    if (!std::isfinite(T[k]))
      return false;
  return std::fabs(T[0]) + std::fabs(T[1]) <= 1.5f && std::fabs(T[4]) + std::fabs(T[5]) <= 1.5f;
}

int dedupe_slots(int F, const uint8_t *const *ptrs, const float *T, const uint8_t **out_ptrs,
                 float *out_T, int *out_w)
{
  int n = 0;
  for (int f = 0; f < F; ++f)
  {
    if (!rigid_enough(T + 12 * f))
      throw CudaError{QM_ERR_INVALID_ARG,
                      "measurement pose is not a rigid transform (finite, rotation rows bounded)"};
    int k = 0;
    while (k < n && !(out_ptrs[k] == ptrs[f] &&
                      std::memcmp(out_T + 12 * k, T + 12 * f, 12 * sizeof(float)) == 0))
      ++k;
    if (k == n)
    {
      out_ptrs[n] = ptrs[f];
      std::memcpy(out_T + 12 * n, T + 12 * f, 12 * sizeof(float));
      out_w[n] = 0;
      ++n;
    }
    out_w[k] += 1;
  }
  return n;
}

std::string validate(const qm_params &p)
{
  if (!bp_supported_d(p.num_hyp))
    return "num_hyp must be one of 32, 48, 64, 96, 128";
  if (p.bp_levels < 1 || p.bp_levels > kMaxLevels)
    return "bp_levels must be in [1, 8]";
  for (int l = 0; l < p.bp_levels; ++l)
    if (p.bp_iters[l] < 0 || p.bp_iters[l] > 1000)
      return "bp_iters out of range";
  if (p.qt_max_level < 1 || p.qt_max_level > 5)
    return "qt_max_level must be in [1, 5]";
  if (p.qt_min_level < 0 || p.qt_min_level > p.qt_max_level)
    return "qt_min_level must be in [0, qt_max_level]";
  if (!(p.inv_depth_step > 0.0) || !(p.min_inv_depth > 0.0))
    return "inverse-depth range must be positive";
  if (!(p.up_sigma > 0.0) || !(p.up_lambda >= 0.0))
    return "upsample sigma/lambda out of range";
  if (p.arith != QM_ARITH_REFERENCE && p.arith != QM_ARITH_IEEE)
    return "arith must be QM_ARITH_REFERENCE or QM_ARITH_IEEE";
  return "";
}

std::string validate(const Shape &s, const qm_params &p)
{
  if (s.W < 16 || s.H < 16 || s.W > kMaxRowLen || s.H > kMaxColLen)
    return "image size must be within [16, 4096] x [16, 2048]";
  if (s.W % 16 != 0 || s.H % 8 != 0)
    return "width must be a multiple of 16 and height of 8 (the upsampler's line chunks)";
  if (!bp_supported_d(s.D))
    return "num_hyp must be one of 32, 48, 64, 96, 128";
  if (s.F < 1 || s.F > kMaxSlots)
    return "num_slots must be in [1, 32]";
  if (!(s.cam.fx > 0.0f) || !(s.cam.fy > 0.0f))
    return "focal lengths must be positive";
  (void)p;
  return "";
}

JobLayout JobLayout::make(const Shape &s, int nlev)
{
  JobLayout L;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t r = o;
    o = align256(o + bytes);
    return r;
  };
  const size_t P = (size_t)s.W * s.H;
  L.off_levels = take(P);
  int w = s.W / 4, h = s.H / 4;
  for (int l = 0; l < kMaxLevels; ++l)
  {
    L.lw[l] = w;
    L.lh[l] = h;
    if (l < nlev)
    {
      const size_t n = (size_t)w * h * s.D * sizeof(float);
      L.off_data[l] = take(n);
      for (int m = 0; m < 4; ++m)
        L.off_msg[l][m] = take(n);
    }
    w = (w + 1) / 2;
    h = (h + 1) / 2;
  }
  L.off_labels = take((size_t)(s.W / 4) * (s.H / 4) * sizeof(int32_t));
  L.off_sparse = take(P * sizeof(float));
  L.off_dense[0] = take(P * sizeof(float));
  L.off_dense[1] = take(P * sizeof(float));
  L.off_rowres = take(P * sizeof(float2));
  L.off_seeds[0] = take(P * sizeof(float4));
  L.off_seeds[1] = take(P * sizeof(float4));
  L.off_zkey = take(P * sizeof(unsigned long long));
  L.off_sdkey = take(P * sizeof(unsigned long long));
  L.bytes = o;
  return L;
}

JobDesc make_job_desc(const Shape &s, const qm_params &p, const JobBuffers &b, int seeds_cur)
{
  JobDesc J;
  std::memset(&J, 0, sizeof(J));
  J.W = s.W;
  J.H = s.H;
  J.D = s.D;
  J.F = s.F;
  J.cw = s.W / 4;
  J.ch = s.H / 4;
  J.fx = s.cam.fx;
  J.fy = s.cam.fy;
  J.cx = s.cam.cx;
  J.cy = s.cam.cy;
  J.min_inv = p.min_inv_depth;
  J.step = p.inv_depth_step;
  J.levels = b.levels;
  J.nlev = p.bp_levels;
  for (int l = 0; l < p.bp_levels; ++l)
  {
    J.lv[l].w = b.lw[l];
    J.lv[l].h = b.lh[l];
    J.lv[l].data = b.data[l];
    for (int m = 0; m < 4; ++m)
      J.lv[l].msg[m] = b.msg[l][m];
  }
  J.labels = b.labels;
  J.sparse = b.sparse;
  J.dense = b.dense[0];
  J.rowres = b.rowres;
  J.seeds_in = b.seeds[seeds_cur];
  J.seeds_out = b.seeds[seeds_cur ^ 1];
  J.zkey = b.zkey;
  J.table = nullptr; // the batched pipeline does not keep the fusion's source table
  for (int k = 0; k < 12; ++k)
    J.Tf[k] = (k == 0 || k == 5 || k == 10) ? 1.0f : 0.0f;
  return J;
}

// Stage table of one job set under one set of launch shapes, with the device
// copy of its block prefixes.
struct TableBuf
{
  StageTable table;
  int *d_prefix = nullptr;
  TableBuf() = default;
  TableBuf(const TableBuf &) = delete;
  TableBuf &operator=(const TableBuf &) = delete;
  ~TableBuf()
  {
    if (d_prefix)
      cudaFree(d_prefix);
  }
};

struct Plan
{
  std::vector<int> active;
  std::unique_ptr<TableBuf> tb;
  bool tuned = false;                  // launch shapes settled (timed or fixed)
  size_t group_bytes = 0;              // the job grouping the graphs were captured with
  int coarse_cells = 0;                // the coarse-level threshold they were captured with
  bool stagger = false;                // the branch staggering they were captured with
  cudaGraphExec_t exec[2] = {nullptr, nullptr}; // by step parity
  StageTable &table() { return tb->table; }
  void drop_graphs()
  {
    for (auto &e : exec)
      if (e)
      {
        cudaGraphExecDestroy(e);
        e = nullptr;
      }
  }
  ~Plan() { drop_graphs(); }
};

std::string validate(const Tune &t, int max_w, int max_h)
{
  auto one_of = [](int v, int a, int b, int c) { return v == a || v == b || v == c; };
  if (!one_of(t.sweep_warps, 4, 8, 16) || !one_of(t.extract_warps, 4, 8, 16))
    return "BP warps per block must be 4, 8 or 16";
  if (!one_of(t.row_warps, 1, 2, 4) || !one_of(t.col_lines, 2, 4, 8))
    return "row-solve rows per block must be 1, 2 or 4 and column-solve lines 2, 4 or 8";
  if (!one_of(t.cost_blocks, 3, 4, 5))
    return "cost-kernel blocks per SM must be 3, 4 or 5";
  if (row_solve_smem(max_w, t.row_warps) > (size_t)kMaxBlockSmem ||
      col_solve_smem(max_h, t.col_lines) > (size_t)kMaxBlockSmem)
    return "line-solver block exceeds the shared memory of a block at this image size";
  return "";
}

Engine::Engine(int device, const qm_params &p, const std::vector<Shape> &shapes)
    : device_(device), params_(p), shapes_(shapes)
{
  std::string err = validate(p);
  if (!err.empty())
    throw CudaError{QM_ERR_INVALID_ARG, err};
  if (shapes.empty())
    throw CudaError{QM_ERR_INVALID_ARG, "no jobs"};
  for (const auto &s : shapes)
  {
    err = validate(s, p);
    if (!err.empty())
      throw CudaError{QM_ERR_INVALID_ARG, err};
  }
  check(cudaSetDevice(device), "cudaSetDevice");
  check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  check(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming), "cudaEventCreate");
  for (int i = 0; i + 1 < kMaxBranches; ++i)
  {
    check(cudaStreamCreateWithFlags(&branch_[i], cudaStreamNonBlocking), "cudaStreamCreate");
    check(cudaEventCreateWithFlags(&ev_join_[i], cudaEventDisableTiming), "cudaEventCreate");
    check(cudaEventCreateWithFlags(&ev_stage_[i], cudaEventDisableTiming), "cudaEventCreate");
  }
  check(cudaEventCreate(&ev0_), "cudaEventCreate");
  check(cudaEventCreate(&ev1_), "cudaEventCreate");
  prepare_upsample_kernels();
  const int n = njobs();
  size_t total = 0;
  std::vector<size_t> base(n);
  for (int j = 0; j < n; ++j)
  {
    layouts_.push_back(JobLayout::make(shapes[j], p.bp_levels));
    base[j] = total;
    total += layouts_[j].bytes;
  }
  check(cudaMalloc(&arena_, total), "device workspace allocation");
  bufs_.resize(n);
  seeds_cur_.assign(n, 0);
  for (int j = 0; j < n; ++j)
  {
    char *b0 = (char *)arena_ + base[j];
    const JobLayout &L = layouts_[j];
    JobBuffers &B = bufs_[j];
    B.levels = (uint8_t *)(b0 + L.off_levels);
    for (int l = 0; l < p.bp_levels; ++l)
    {
      B.data[l] = (float *)(b0 + L.off_data[l]);
      for (int m = 0; m < 4; ++m)
        B.msg[l][m] = (float *)(b0 + L.off_msg[l][m]);
    }
    for (int l = 0; l < kMaxLevels; ++l)
    {
      B.lw[l] = L.lw[l];
      B.lh[l] = L.lh[l];
    }
    B.labels = (int32_t *)(b0 + L.off_labels);
    B.sparse = (float *)(b0 + L.off_sparse);
    B.dense[0] = (float *)(b0 + L.off_dense[0]);
    B.dense[1] = (float *)(b0 + L.off_dense[1]);
    B.rowres = (float2 *)(b0 + L.off_rowres);
    B.seeds[0] = (float4 *)(b0 + L.off_seeds[0]);
    B.seeds[1] = (float4 *)(b0 + L.off_seeds[1]);
    B.zkey = (unsigned long long *)(b0 + L.off_zkey);
    B.sdkey = (unsigned long long *)(b0 + L.off_sdkey);
    const size_t P = (size_t)shapes[j].W * shapes[j].H;
    check(cudaMemsetAsync(B.seeds[0], 0, P * sizeof(float4) * 1, stream_), "memset");
    check(cudaMemsetAsync(B.seeds[1], 0, P * sizeof(float4) * 1, stream_), "memset");
    check(cudaMemsetAsync(B.zkey, 0xff, P * sizeof(unsigned long long), stream_), "memset");
    check(cudaMemsetAsync(B.sdkey, 0xff, P * sizeof(unsigned long long), stream_), "memset");
    check(cudaMemsetAsync(B.sparse, 0, P * sizeof(float), stream_), "memset");
    check(cudaMemsetAsync(B.dense[0], 0, P * sizeof(float), stream_), "memset");
    check(cudaMemsetAsync(B.dense[1], 0, P * sizeof(float), stream_), "memset");
  }
  slot_base_.resize(n);
  for (int j = 0; j < n; ++j)
  {
    slot_base_[j] = total_slots_;
    total_slots_ += shapes[j].F;
  }
  for (int q = 0; q < 2; ++q)
  {
    check(cudaHostAlloc((void **)&h_slot_ptr_[q], sizeof(void *) * total_slots_,
                        cudaHostAllocDefault),
          "pinned allocation");
    check(cudaHostAlloc((void **)&h_slot_T_[q], sizeof(float) * 12 * total_slots_,
                        cudaHostAllocDefault),
          "pinned allocation");
    check(cudaHostAlloc((void **)&h_slot_w_[q], sizeof(int) * total_slots_, cudaHostAllocDefault),
          "pinned allocation");
    std::memset(h_slot_ptr_[q], 0, sizeof(void *) * total_slots_);
    std::memset(h_slot_T_[q], 0, sizeof(float) * 12 * total_slots_);
    std::memset(h_slot_w_[q], 0, sizeof(int) * total_slots_);
    check(cudaHostAlloc((void **)&h_run_[q], sizeof(JobDesc) * n, cudaHostAllocDefault),
          "pinned allocation");
  }
  check(cudaMalloc((void **)&d_slot_ptr_, sizeof(void *) * total_slots_), "device allocation");
  check(cudaMalloc((void **)&d_slot_T_, sizeof(float) * 12 * total_slots_), "device allocation");
  check(cudaMalloc((void **)&d_slot_w_, sizeof(int) * total_slots_), "device allocation");
  master_.resize(n);
  for (int j = 0; j < n; ++j)
  {
    master_[j] = make_job_desc(shapes[j], p, bufs_[j], 0);
    master_[j].slot_base = slot_base_[j];
  }
  check(cudaMalloc((void **)&d_run_, sizeof(JobDesc) * n), "device allocation");
  check(cudaStreamSynchronize(stream_), "engine init");
}

Engine::~Engine()
{
  cudaSetDevice(device_);
  if (stream_)
    cudaStreamSynchronize(stream_);
  plans_.clear();
  if (arena_)
    cudaFree(arena_);
  if (d_slot_ptr_)
    cudaFree(d_slot_ptr_);
  if (d_slot_T_)
    cudaFree(d_slot_T_);
  if (d_slot_w_)
    cudaFree(d_slot_w_);
  if (d_run_)
    cudaFree(d_run_);
  for (int q = 0; q < 2; ++q)
  {
    if (h_slot_ptr_[q])
      cudaFreeHost(h_slot_ptr_[q]);
    if (h_slot_T_[q])
      cudaFreeHost(h_slot_T_[q]);
    if (h_slot_w_[q])
      cudaFreeHost(h_slot_w_[q]);
    if (h_run_[q])
      cudaFreeHost(h_run_[q]);
  }
  if (ev0_)
    cudaEventDestroy(ev0_);
  if (ev1_)
    cudaEventDestroy(ev1_);
  for (int i = 0; i + 1 < kMaxBranches; ++i)
  {
    if (branch_[i])
    {
      cudaStreamSynchronize(branch_[i]);
      cudaStreamDestroy(branch_[i]);
    }
    if (ev_join_[i])
      cudaEventDestroy(ev_join_[i]);
    if (ev_stage_[i])
      cudaEventDestroy(ev_stage_[i]);
  }
  if (ev_fork_)
    cudaEventDestroy(ev_fork_);
  if (stream_)
    cudaStreamDestroy(stream_);
}

void Engine::set_inputs(int j, const uint8_t *ref, int ref_pitch, const uint8_t *const *slots,
                        int slot_pitch, const float *T_slot_ref, const float *T_fuse)
{
  JobDesc &J = master_[j];
  J.ref = ref;
  J.ref_pitch = ref_pitch;
  J.slot_pitch = slot_pitch;
  const int b = slot_base_[j];
  const int q = parity_;
  J.F = dedupe_slots(shapes_[j].F, slots, T_slot_ref, h_slot_ptr_[q] + b, h_slot_T_[q] + 12 * b,
                     h_slot_w_[q] + b);
  if (T_fuse)
    std::memcpy(J.Tf, T_fuse, 12 * sizeof(float));
}

void Engine::reset_seeds(int j)
{
  const size_t P = (size_t)shapes_[j].W * shapes_[j].H;
  check(cudaMemsetAsync(bufs_[j].seeds[0], 0, P * sizeof(float4), stream_), "memset");
  check(cudaMemsetAsync(bufs_[j].seeds[1], 0, P * sizeof(float4), stream_), "memset");
  check(cudaStreamSynchronize(stream_), "reset seeds");
  seeds_cur_[j] = 0;
}

std::unique_ptr<TableBuf> Engine::build_table(const std::vector<int> &active, const Tune &tune)
{
  auto tb = std::make_unique<TableBuf>();
  const int L = params_.bp_levels;
  const int n = (int)active.size();
  std::vector<std::vector<int>> per_job;
  std::vector<int> ds;
  StageTable &T = tb->table;
  T.tune = tune;
  for (int i = 0; i < n; ++i)
  {
    const int j = active[i];
    ds.push_back(shapes_[j].D);
    T.max_w = std::max(T.max_w, shapes_[j].W);
    T.max_h = std::max(T.max_h, shapes_[j].H);
    per_job.push_back(stage_blocks(shapes_[j], layouts_[j], params_, tune));
    for (int l = 0; l < L; ++l)
      T.level_bytes.push_back((size_t)5 * layouts_[j].lw[l] * layouts_[j].lh[l] * shapes_[j].D *
                              sizeof(float));
    T.level_cells.resize(L, 0);
    for (int l = 0; l < L; ++l)
      T.level_cells[l] = std::max(T.level_cells[l], (long)layouts_[j].lw[l] * layouts_[j].lh[l]);
  }
  T.add_jobs(per_job, ds);
  const int ns = (int)T.uniform.size();
  check(cudaMalloc((void **)&tb->d_prefix, sizeof(int) * T.hprefix.size()), "device allocation");
  check(cudaMemcpy(tb->d_prefix, T.hprefix.data(), sizeof(int) * T.hprefix.size(),
                   cudaMemcpyHostToDevice),
        "plan upload");
  for (int st = 0; st < ns; ++st)
    T.prefix.push_back(tb->d_prefix + (size_t)st * (n + 1));
  return tb;
}

Plan &Engine::plan_for(const std::vector<int> &active)
{
  auto it = plans_.find(active);
  if (it != plans_.end())
  {
    Plan &pl = *it->second;
    if (pl.group_bytes != group_bytes_ || pl.coarse_cells != coarse_cells_ ||
        pl.stagger != stagger_)
      pl.drop_graphs();
    return pl;
  }
  auto pl = std::make_unique<Plan>();
  pl->active = active;
  int max_w = 0, max_h = 0;
  for (int j : active)
  {
    max_w = std::max(max_w, shapes_[j].W);
    max_h = std::max(max_h, shapes_[j].H);
  }
  // a fixed shape that does not fit this set's lines falls back to the
  // defaults (which fit every valid image size)
  Tune t = fixed_tune_;
  if (!validate(t, max_w, max_h).empty())
    t = Tune{};
  pl->tb = build_table(active, t);
  pl->tuned = !autotune_;
  Plan &ref = *pl;
  plans_[active] = std::move(pl);
  return ref;
}

// Candidate c (0..2) of every launch-shape family; a line-solver candidate
// that does not fit the set's longest line keeps the default.
static Tune candidate(int c, int max_w, int max_h)
{
  static const int kWarps[3] = {4, 8, 16}, kRows[3] = {1, 2, 4}, kCols[3] = {2, 4, 8};
  static const int kCostB[3] = {4, kCostBlocks, 3};
  Tune t;
  t.sweep_warps = t.extract_warps = kWarps[c];
  t.cost_blocks = kCostB[c];
  if (row_solve_smem(max_w, kRows[c]) <= (size_t)kMaxBlockSmem)
    t.row_warps = kRows[c];
  if (col_solve_smem(max_h, kCols[c]) <= (size_t)kMaxBlockSmem)
    t.col_lines = kCols[c];
  return t;
}

void Engine::tune_plan(Plan &pl)
{
  // The candidates of the five families are timed side by side: run c uses
  // candidate c of each, and every family keeps its fastest candidate by the
  // summed device time of its launches.  Runs are eager, with an event pair
  // around every launch; the first run warms the caches and is not counted,
  // then each candidate runs twice and keeps its lower time.  A run writes
  // the same buffers as the real run that follows (it reads the same seeds
  // and inputs), so tuning changes no result.
  const StageTable &T0 = pl.table();
  std::unique_ptr<TableBuf> cand[3];
  for (int c = 0; c < 3; ++c)
    cand[c] = build_table(pl.active, candidate(c, T0.max_w, T0.max_h));
  const Batch B = upload((int)pl.active.size(), stream_);
  const Stages st{params_.bp_levels};
  const int fam_kind[5] = {kSweep, kExtract, kRowSolve, kColSolve, kCost};
  float best[3][5];
  for (auto &r : best)
    for (float &v : r)
      v = INFINITY;
  const int order[7] = {1, 0, 1, 2, 0, 1, 2};
  for (int r = 0; r < 7; ++r)
  {
    const int c = order[r];
    LaunchProfile prof;
    float ms[kNumKinds] = {};
    try
    {
      enqueue_range(B, cand[c]->table, params_, group_bytes_, coarse_cells_, 0, st.count() - 1,
                    stream_, &prof);
      check(cudaStreamSynchronize(stream_), "autotune run");
    }
    catch (...)
    {
      for (auto &m : prof.marks)
      {
        cudaEventDestroy(m.e0);
        cudaEventDestroy(m.e1);
      }
      throw;
    }
    for (auto &m : prof.marks)
    {
      float t = 0.0f;
      cudaEventElapsedTime(&t, m.e0, m.e1);
      ms[m.kind] += t;
      cudaEventDestroy(m.e0);
      cudaEventDestroy(m.e1);
    }
    if (r > 0)
      for (int f = 0; f < 5; ++f)
        best[c][f] = std::min(best[c][f], ms[fam_kind[f]]);
  }
  int pick[5];
  for (int f = 0; f < 5; ++f)
  {
    pick[f] = 1;
    for (int c = 0; c < 3; ++c)
      if (best[c][f] < best[pick[f]][f])
        pick[f] = c;
  }
  Tune t;
  t.sweep_warps = cand[pick[0]]->table.tune.sweep_warps;
  t.extract_warps = cand[pick[1]]->table.tune.extract_warps;
  t.row_warps = cand[pick[2]]->table.tune.row_warps;
  t.col_lines = cand[pick[3]]->table.tune.col_lines;
  t.cost_blocks = cand[pick[4]]->table.tune.cost_blocks;
  pl.drop_graphs();
  pl.tb = build_table(pl.active, t);
  pl.tuned = true;
}

void Engine::set_branches(int k)
{
  k = std::max(1, std::min(k, kMaxBranches));
  if (k == branches_)
    return;
  check(cudaSetDevice(device_), "cudaSetDevice");
  check(cudaStreamSynchronize(stream_), "branch switch");
  branches_ = k;
  plans_.clear();
}

void Engine::set_autotune(bool on)
{
  check(cudaSetDevice(device_), "cudaSetDevice");
  check(cudaStreamSynchronize(stream_), "autotune switch");
  autotune_ = on;
  plans_.clear();
}

void Engine::set_tune(const Tune &t)
{
  int max_w = 0, max_h = 0;
  for (const auto &s : shapes_)
  {
    max_w = std::max(max_w, s.W);
    max_h = std::max(max_h, s.H);
  }
  const std::string err = validate(t, max_w, max_h);
  if (!err.empty())
    throw CudaError{QM_ERR_INVALID_ARG, err};
  check(cudaSetDevice(device_), "cudaSetDevice");
  check(cudaStreamSynchronize(stream_), "launch-shape switch");
  fixed_tune_ = t;
  autotune_ = false;
  plans_.clear();
}

void Engine::pack(const std::vector<int> &active)
{
  for (size_t i = 0; i < active.size(); ++i)
  {
    const int j = active[i];
    JobDesc J = master_[j];
    J.seeds_in = bufs_[j].seeds[seeds_cur_[j]];
    J.seeds_out = bufs_[j].seeds[seeds_cur_[j] ^ 1];
    J.dense = bufs_[j].dense[parity_];
    h_run_[parity_][i] = J;
  }
}

Batch Engine::upload(int n, cudaStream_t s)
{
  const int q = parity_;
  check(cudaMemcpyAsync(d_run_, h_run_[q], sizeof(JobDesc) * n, cudaMemcpyHostToDevice, s),
        "descriptor upload");
  check(cudaMemcpyAsync(d_slot_ptr_, h_slot_ptr_[q], sizeof(void *) * total_slots_,
                        cudaMemcpyHostToDevice, s),
        "slot upload");
  check(cudaMemcpyAsync(d_slot_T_, h_slot_T_[q], sizeof(float) * 12 * total_slots_,
                        cudaMemcpyHostToDevice, s),
        "slot upload");
  check(cudaMemcpyAsync(d_slot_w_, h_slot_w_[q], sizeof(int) * total_slots_,
                        cudaMemcpyHostToDevice, s),
        "slot upload");
  Batch B;
  std::memset(&B, 0, sizeof(B));
  B.jobs = d_run_;
  B.njobs = n;
  B.slot_ptr = d_slot_ptr_;
  B.slot_T = d_slot_T_;
  B.slot_w = d_slot_w_;
  return B;
}

int Engine::enqueue(Plan &pl, cudaStream_t s)
{
  const Batch B = upload((int)pl.active.size(), s);
  const Stages st{params_.bp_levels};
  pl.group_bytes = group_bytes_;
  pl.coarse_cells = coarse_cells_;
  pl.stagger = stagger_;
  const int n = (int)pl.active.size();
  const int k = std::min(branches_, n);
  if (k < 2)
    return enqueue_range(B, pl.table(), params_, group_bytes_, coarse_cells_, 0, st.count() - 1,
                         s);
  // k independent branches over consecutive ranges of the jobs (every stage
  // is per job): the GPU fills the latency-bound stretches of one branch
  // (coarse BP levels, line solves) with the other branches' work
  // Staggered (optional): branch i + 1 starts when branch i's cost volume
  // is done, so that cost kernels (bound by instruction issue) run beside
  // the previous branch's BP half-sweeps (bound by HBM bandwidth) instead of
  // beside each other.
  check(cudaEventRecord(ev_fork_, s), "fork");
  int nl = 0;
  for (int i = 0; i < k; ++i)
  {
    cudaStream_t bs = i == 0 ? s : branch_[i - 1];
    const int ja = n * i / k, jb = n * (i + 1) / k;
    if (i > 0)
      check(cudaStreamWaitEvent(bs, stagger_ ? ev_stage_[i - 1] : ev_fork_, 0), "fork");
    if (stagger_ && i + 1 < k)
    {
      nl += enqueue_range(B, pl.table(), params_, group_bytes_, coarse_cells_, 0, st.cost(), bs,
                          nullptr, ja, jb);
      check(cudaEventRecord(ev_stage_[i], bs), "stage");
      nl += enqueue_range(B, pl.table(), params_, group_bytes_, coarse_cells_, st.cost() + 1,
                          st.count() - 1, bs, nullptr, ja, jb);
    }
    else
      nl += enqueue_range(B, pl.table(), params_, group_bytes_, coarse_cells_, 0, st.count() - 1,
                          bs, nullptr, ja, jb);
  }
  for (int i = 1; i < k; ++i)
  {
    check(cudaEventRecord(ev_join_[i - 1], branch_[i - 1]), "join");
    check(cudaStreamWaitEvent(s, ev_join_[i - 1], 0), "join");
  }
  return nl;
}

void Engine::run(const std::vector<int> &active)
{
  launch(active);
  check(cudaStreamSynchronize(stream_), "pipeline run");
}

void Engine::launch(const std::vector<int> &active)
{
  if (active.empty())
    return;
  check(cudaSetDevice(device_), "cudaSetDevice");
  Plan &pl = plan_for(active);
  pack(active);
  if (!pl.tuned)
    tune_plan(pl);
  last_tune_ = pl.table().tune;
  if (graphs_)
  {
    // one graph per parity: its memcpy nodes read that parity's pinned
    // descriptor and slot tables
    cudaGraphExec_t &exec = pl.exec[parity_];
    if (!exec)
    {
      cudaGraph_t g = nullptr;
      check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "graph capture");
      int nl = 0;
      try
      {
        nl = enqueue(pl, stream_);
      }
      catch (...)
      {
        cudaStreamEndCapture(stream_, &g);
        if (g)
          cudaGraphDestroy(g);
        throw;
      }
      check(cudaStreamEndCapture(stream_, &g), "graph capture");
      const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
      cudaGraphDestroy(g);
      check(e, "graph instantiate");
      last_launches_ = nl;
    }
    check(cudaEventRecord(ev0_, stream_), "event");
    check(cudaGraphLaunch(exec, stream_), "graph launch");
    check(cudaEventRecord(ev1_, stream_), "event");
  }
  else
  {
    check(cudaEventRecord(ev0_, stream_), "event");
    last_launches_ = enqueue(pl, stream_);
    check(cudaEventRecord(ev1_, stream_), "event");
  }
  for (int j : active)
    seeds_cur_[j] ^= 1;
}

float Engine::last_run_ms() const
{
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, ev0_, ev1_);
  return ms;
}

void Engine::profile(const std::vector<int> &active, float *ms, int *launches)
{
  check(cudaSetDevice(device_), "cudaSetDevice");
  Plan &pl = plan_for(active);
  pack(active);
  if (!pl.tuned)
    tune_plan(pl);
  last_tune_ = pl.table().tune;
  const Batch B = upload((int)pl.active.size(), stream_);
  const Stages st{params_.bp_levels};
  LaunchProfile prof;
  try
  {
    enqueue_range(B, pl.table(), params_, group_bytes_, coarse_cells_, 0, st.count() - 1, stream_,
                  &prof);
    check(cudaStreamSynchronize(stream_), "profile run");
  }
  catch (...)
  {
    for (auto &m : prof.marks)
    {
      cudaEventDestroy(m.e0);
      cudaEventDestroy(m.e1);
    }
    throw;
  }
  for (int k = 0; k < kNumKinds; ++k)
  {
    ms[k] = 0.0f;
    launches[k] = 0;
  }
  for (auto &m : prof.marks)
  {
    float t = 0.0f;
    cudaEventElapsedTime(&t, m.e0, m.e1);
    ms[m.kind] += t;
    launches[m.kind] += 1;
    cudaEventDestroy(m.e0);
    cudaEventDestroy(m.e1);
  }
  for (int j : active)
    seeds_cur_[j] ^= 1;
}

// ---------------------------------------------------------------------------
// Single-keyframe stage calls (C-ABI stage entry points).

namespace stage
{

Batch single(const JobDesc &J)
{
  Batch B;
  std::memset(&B, 0, sizeof(B));
  B.jobs = nullptr;
  B.njobs = 1;
  B.one = J;
  return B;
}

int run_range(const Batch &B, const Shape &s, const qm_params &p, int first, int last,
              cudaStream_t stream)
{
  const JobLayout lay = JobLayout::make(s, p.bp_levels);
  StageTable T;
  T.add_jobs({stage_blocks(s, lay, p, T.tune)}, {s.D});
  T.max_w = s.W;
  T.max_h = s.H;
  for (int l = 0; l < p.bp_levels; ++l)
    T.level_cells.push_back((long)lay.lw[l] * lay.lh[l]);
  return enqueue_range(B, T, p, 0, QM_DEFAULT_COARSE_CELLS, first, last, stream);
}

int first_of(const char *name, int L)
{
  const Stages st{L};
  const std::string n(name);
  if (n == "quadtree")
    return st.qt();
  if (n == "cost")
    return st.cost();
  if (n == "bp")
    return L > 1 ? st.pyr(1) : st.inherit(0);
  if (n == "upsample")
    return st.row();
  if (n == "fuse")
    return st.ftrans();
  return -1;
}

int last_of(const char *name, int L)
{
  const Stages st{L};
  const std::string n(name);
  if (n == "quadtree")
    return st.qt();
  if (n == "cost")
    return st.cost();
  if (n == "bp")
    return st.extract();
  if (n == "upsample")
    return st.col();
  if (n == "fuse")
    return st.fupd();
  return -1;
}

} // namespace stage

} // namespace qm
