// Host engine of the dense pipeline: owns the device buffers of N keyframe
// jobs and runs quadtree -> cost -> BP -> extraction -> upsampling -> fusion
// for any subset of them, one kernel launch per stage, optionally replayed
// from a captured CUDA graph.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "launch.h"

namespace qm
{

// thread-local error message behind qm_last_error()
void set_error(const std::string &msg);
const char *get_error();

struct CudaError
{
  int status;
  std::string msg;
};

// throws CudaError on failure
void check(cudaError_t e, const char *what);

// Kernel kinds, for per-kind timing (qm_batch_profile).
enum KernelKind
{
  kQuadtree = 0,
  kCost,
  kPyramid,
  kMsgInit, // levels with fewer than two half-sweeps only
  kSweep,
  kExtract,
  kRowSolve,
  kColSolve,
  kFuseTransform,
  kFuseFill, // not launched (hole filling runs inside kFuseUpdate); keeps the
             // kind indices of qm_batch_profile stable
  kFuseUpdate,
  kNumKinds
};

// Default L2 budget of a BP job range: 0, every level over all jobs at once.
// Ranges that fit in L2 (e.g. 64 MiB) keep a range's costs and messages
// resident between its half-sweeps, but on a B200 the smaller launches lose
// more to tails and launch gaps than L2 residency saves (752x480, 64
// hypotheses, 32 streams: 4.60 ms per batch ungrouped, 4.72 ms at 64 MiB,
// 5.23 ms at 24 MiB).
constexpr size_t kDefaultGroupBytes = 0;

// Default number of concurrent pipeline branches per batch: two (the halves
// of the active jobs as independent graph branches) measured 3 % faster than
// one sequence at 32 streams of 752x480 (3.27 vs 3.37 ms per batch), with
// bit-identical results.
// Default coarse-level threshold of the BP: the top pyramid levels whose
// largest cell count over the active jobs is at most this run all their
// half-sweeps in one cluster launch (k_bp_coarse) instead of one launch per
// half-sweep; 0 disables it.  4096 takes levels 2 and 3 of a 752x480 or
// 1280x720 keyframe (1410 / 360 and 3600 / 920 cells) and level 3 of a
// 1920x1080 one.
#ifndef QM_DEFAULT_COARSE_CELLS
#define QM_DEFAULT_COARSE_CELLS 4096
#endif

#ifndef QM_DEFAULT_BRANCHES
#define QM_DEFAULT_BRANCHES 2
#endif
constexpr int kMaxBranches = 4;

struct LaunchProfile
{
  struct Mark
  {
    int kind;
    cudaEvent_t e0, e1;
  };
  std::vector<Mark> marks;
};

struct Shape
{
  int W, H, D, F;
  Cam cam;
};

struct JobBuffers
{
  uint8_t *levels = nullptr;
  float *data[kMaxLevels] = {};
  float *msg[kMaxLevels][4] = {};
  int lw[kMaxLevels] = {}, lh[kMaxLevels] = {};
  int32_t *labels = nullptr;
  float *sparse = nullptr;
  float *dense[2] = {}; // by step parity (a step's result can be read
                        // back while the next step runs)
  float2 *rowres = nullptr;
  float4 *seeds[2] = {};
  unsigned long long *zkey = nullptr;  // fusion z-buffer (reset by the row solve)
  unsigned long long *sdkey = nullptr; // semi-dense z-buffer (all ones between its steps)
};

// Byte layout of one job's buffers (offsets from a 256-byte aligned base).
struct JobLayout
{
  size_t bytes = 0;
  size_t off_levels, off_data[kMaxLevels], off_msg[kMaxLevels][4], off_labels, off_sparse,
      off_dense[2], off_rowres, off_seeds[2], off_zkey, off_sdkey;
  int lw[kMaxLevels], lh[kMaxLevels];
  static JobLayout make(const Shape &s, int nlev);
};

// Fills a JobDesc (geometry, parameters, buffer pointers) for one job.
JobDesc make_job_desc(const Shape &s, const qm_params &p, const JobBuffers &b, int seeds_cur);

// Validates a parameter struct and a shape; returns an empty string when OK.
std::string validate(const qm_params &p);
std::string validate(const Shape &s, const qm_params &p);

KParams kparams(const qm_params &p);

// True when the 3x4 pose is finite and its rotation rows satisfy
// |r00| + |r01| <= 1.5 and |r10| + |r11| <= 1.5 (every rotation does): the
// cost kernel's rotated 3x3 patch then stays inside the measurement image.
bool rigid_enough(const float *T);

// Merges measurement slots with the same image and pose: writes the unique
// slots (first-occurrence order) with their multiplicities and returns how
// many there are.  Throws CudaError(QM_ERR_INVALID_ARG) for a pose that is
// not rigid_enough.
int dedupe_slots(int F, const uint8_t *const *ptrs, const float *T, const uint8_t **out_ptrs,
                 float *out_T, int *out_w);

// Stage plan of one active job set: block prefix per stage, in one device
// buffer, plus the captured graph.
struct Plan;
struct TableBuf;

// Validates launch shapes for lines up to max_w / max_h samples.
std::string validate(const Tune &t, int max_w, int max_h);

class Engine
{
public:
  Engine(int device, const qm_params &p, const std::vector<Shape> &shapes);
  ~Engine();
  Engine(const Engine &) = delete;
  Engine &operator=(const Engine &) = delete;

  int njobs() const { return (int)shapes_.size(); }
  const Shape &shape(int j) const { return shapes_[j]; }
  const JobBuffers &buffers(int j) const { return bufs_[j]; }
  const qm_params &params() const { return params_; }
  cudaStream_t stream() const { return stream_; }
  int device() const { return device_; }

  // Step parity: selects the output buffer and the pinned descriptor and
  // slot tables that set_inputs / launch use, so that the host can prepare
  // step t+1 while step t (the other parity) is still in flight.
  void set_parity(int p) { parity_ = p & 1; }
  int parity() const { return parity_; }
  // fused depth buffer of job j for the current parity
  float *dense(int j) const { return bufs_[j].dense[parity_]; }

  // Inputs of job j for the next run.  Device pointers; T_slot_ref is
  // F*12 floats (host), T_fuse 12 floats T_income<-lastfuse (host).
  void set_inputs(int j, const uint8_t *ref, int ref_pitch, const uint8_t *const *slots,
                  int slot_pitch, const float *T_slot_ref, const float *T_fuse);
  // Current seed buffer of job j (after the last run).
  float4 *seeds(int j) const { return bufs_[j].seeds[seeds_cur_[j]]; }
  void reset_seeds(int j);

  // Enqueues the pipeline for `active` job indices on stream() without
  // waiting.  Throws CudaError.  Graph capture is used when `graphs` is set.
  void launch(const std::vector<int> &active);
  // launch() and wait for it
  void run(const std::vector<int> &active);
  void set_graphs(bool on) { graphs_ = on; }
  // L2 budget of a BP job range (0: every level over all jobs at once)
  void set_group_bytes(size_t bytes) { group_bytes_ = bytes; }
  // k (1..4): the pipeline runs as k concurrent branches over consecutive
  // ranges of the active jobs (graph branches, or streams when launching
  // eagerly); 1: one sequence over all jobs.  Results do not depend on it.
  void set_branches(int k);
  int branches() const { return branches_; }
  size_t group_bytes() const { return group_bytes_; }
  // coarse BP levels (at most `cells` cells in every active job) in one
  // cluster launch; 0: one launch per half-sweep at every level.  Results
  // do not depend on it.
  void set_coarse_cells(int cells) { coarse_cells_ = cells < 0 ? 0 : cells; }
  // true: branch i + 1 starts once branch i's cost volume is done, so the
  // issue-bound cost kernel of one branch runs beside the bandwidth-bound
  // BP of the previous one; false (the default; measured faster on a B200:
  // 2.91 vs 2.97 ms per 32 x 752x480 batch with two branches): all
  // branches start together.  Results do not depend on it.
  void set_stagger(bool on) { stagger_ = on; }
  bool stagger() const { return stagger_; }
  int coarse_cells() const { return coarse_cells_; }
  int last_launches() const { return last_launches_; }
  // 1: the sparse buffers arrive filled with the semi-dense tracker's depths
  // (the quadtree pass keeps them instead of clearing)
  void set_keep_sparse(bool on)
  {
    for (auto &J : master_)
      J.keep_sparse = on ? 1 : 0;
  }
  // Launch shapes of the BP and line-solver kernels.  With autotune on (the
  // default) each active job set times three candidates per kernel family
  // on its first run and keeps the fastest; set_tune fixes the shapes for
  // every set (autotune off).  Results do not depend on the shapes.
  void set_autotune(bool on);
  bool autotune() const { return autotune_; }
  void set_tune(const Tune &t);
  // shapes of the last launched or profiled set
  Tune last_tune() const { return last_tune_; }
  // Events bracketing the device work of the last run (for timing).
  float last_run_ms() const;
  // Runs the pipeline once with eager launches, each bracketed by events;
  // ms[k] / launches[k] receive the summed device time and launch count per
  // KernelKind.
  void profile(const std::vector<int> &active, float *ms, int *launches);

private:
  Plan &plan_for(const std::vector<int> &active);
  std::unique_ptr<TableBuf> build_table(const std::vector<int> &active, const Tune &tune);
  void tune_plan(Plan &pl);
  // packs the descriptors of `active` into the pinned run array
  void pack(const std::vector<int> &active);
  // enqueues the descriptor and slot-table uploads; returns the batch
  Batch upload(int n, cudaStream_t s);
  int enqueue(Plan &pl, cudaStream_t s);

  int device_;
  qm_params params_;
  std::vector<Shape> shapes_;
  std::vector<JobLayout> layouts_;
  std::vector<JobBuffers> bufs_;
  std::vector<int> seeds_cur_;
  void *arena_ = nullptr;
  // slot tables (all jobs), pinned host + device
  std::vector<int> slot_base_;
  int total_slots_ = 0;
  const uint8_t **h_slot_ptr_[2] = {};
  float *h_slot_T_[2] = {};
  int *h_slot_w_[2] = {};
  const uint8_t **d_slot_ptr_ = nullptr;
  float *d_slot_T_ = nullptr;
  int *d_slot_w_ = nullptr;
  // job descriptors: host master copy and the packed run arrays
  std::vector<JobDesc> master_;
  JobDesc *h_run_[2] = {};
  JobDesc *d_run_ = nullptr;
  cudaStream_t stream_ = nullptr;
  cudaStream_t branch_[kMaxBranches - 1] = {}; // streams of branches 2..k
  cudaEvent_t ev_fork_ = nullptr, ev_join_[kMaxBranches - 1] = {};
  cudaEvent_t ev_stage_[kMaxBranches - 1] = {}; // branch i's cost stage done
  bool stagger_ = false;
  int branches_ = QM_DEFAULT_BRANCHES;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  bool graphs_ = true;
  int parity_ = 0;
  size_t group_bytes_ = kDefaultGroupBytes;
  int coarse_cells_ = QM_DEFAULT_COARSE_CELLS;
  int last_launches_ = 0;
  bool autotune_ = true;
  Tune fixed_tune_, last_tune_;
  std::map<std::vector<int>, std::unique_ptr<Plan>> plans_;
};

} // namespace qm
