/*
 * C-ABI of the B200-native per-keyframe depth pipeline (libqm_b200.so).
 *
 * Drop-in boundary for QuadtreeMapping's quadmap::Depthmap
 * (include/quadmap/depthmap.h:31-89 of open_quadtree_mapping) and for the
 * device stages behind it (SeedMatrix::extract_depth and fuse_output_depth,
 * src/seed_matrix.cu:448-597).  Plain C: pointers, sizes and status codes;
 * nothing throws across this boundary and no C++ or framework type appears
 * in a signature.  include/qm_depthmap.hpp wraps it in the reference's C++
 * class API.
 *
 * Conventions
 *  - Every function returns a qm_status; qm_last_error() returns a
 *    thread-local message for the last failure on the calling thread.
 *  - Images are 8-bit grayscale, row pitch in BYTES.  Float maps are
 *    row-major with a pitch in ELEMENTS where one is taken.
 *  - Poses are 3x4 row-major float rigid transforms [R | t] as the
 *    reference's SE3<float> stores them (se3.cuh:174, data(r, c) =
 *    data[4r + c]); T_a_b maps points from frame b into frame a.
 *  - Stage entry points take DEVICE pointers and a cudaStream_t passed as
 *    void* (NULL = legacy default stream) and are asynchronous on it.
 *    Facade and batch entry points take HOST buffers and are synchronous.
 *  - Invalid fused depth is -1 (depth_fusion.cu:207-210).
 */
#ifndef QM_CAPI_H
#define QM_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum qm_status {
  QM_OK = 0,
  QM_ERR_INVALID_ARG = 1, /* bad size, pointer, parameter */
  QM_ERR_CUDA = 2,        /* a CUDA runtime call or kernel failed */
  QM_ERR_NO_MEMORY = 3,   /* device or pinned allocation failed */
  QM_ERR_STATE = 4,       /* call not valid in the object's current state */
  QM_ERR_TIMEOUT = 5,     /* a bounded device wait gave up (error flag set) */
  QM_ERR_WORKSPACE = 6    /* caller workspace too small */
} qm_status;

#define QM_MAX_BP_LEVELS 8
#define QM_MAX_SLOTS 32     /* measurement slots per keyframe */
#define QM_RING_CAPACITY 60 /* KEYFRAME_NUM, frameelement.cuh:9 */

enum { QM_ARITH_REFERENCE = 0, QM_ARITH_IEEE = 1 };

/* Algorithm parameters.  qm_params_default() gives the reference's compiled
 * constants: DEPTH_NUM 64 (pixel_cost.cuh:4), MIN_INV_DEPTH 0.01 and
 * STEP_INV_DEPTH (2.0-0.01)/63.0 (stereo_parameter.cuh:5-7), P1 0.003,
 * P2 0.01 (bpextract.cu:222-223), 4 BP levels with {4,10,10,10} half-sweeps
 * fine to coarse (bpextract.cu:41-45), quadtree max level 4, min level 2,
 * threshold 10 (quadtree.cu:40,59,74), upsample sigma 400 and lambda 10
 * (stereo_parameter.cuh upsample_sigma/upsample_lambda).
 * arith: QM_ARITH_REFERENCE computes the projections and normalisations with
 * the reference build's fast-math arithmetic (bit-exact costs and labels
 * versus the reference kernels); QM_ARITH_IEEE uses IEEE-rounded operations
 * (bit-exact versus the CPU oracle). */
typedef struct qm_params {
  int num_hyp;
  double min_inv_depth;
  double inv_depth_step;
  float P1, P2;
  int bp_levels;
  int bp_iters[QM_MAX_BP_LEVELS]; /* fine -> coarse */
  int qt_max_level;
  int qt_min_level;
  float qt_threshold;
  double up_sigma;
  double up_lambda;
  int arith;
} qm_params;

typedef struct qm_camera {
  float fx, fy, cx, cy; /* PinholeCamera order (pinhole_camera.cuh:42) */
} qm_camera;

/* ---------------------------------------------------------------- misc */
void qm_params_default(qm_params *p);
const char *qm_last_error(void);
int qm_version(void); /* major*10000 + minor*100 + patch */

/* ------------------------------------------------- Depthmap facade ----
 * quadmap::Depthmap (depthmap.h:34-75, depthmap.cpp:19-68).  One camera
 * stream: frame ring, frame-selection policy of SeedMatrix::add_frames
 * (seed_matrix.cu:106-209), dense extraction and fusion.  The semi-dense
 * tracker (seed_matrix.cu:120-140) is built but off by default: until
 * qm_depthmap_set_semidense(h, 1) the upsampler's sparse input and the debug
 * map hold the BP node depths only; with it on, the tracker's projected
 * depths join them as in the reference.  With the tracker on, results agree
 * with the reference's own tracker kernels but are not identical to them:
 * the reference resolves pixel collisions and in-place neighbourhood passes
 * by thread scheduling, this library by fixed rules (nearest wins, Jacobi
 * passes).  The image is expected undistorted (the reference's host
 * cv::remap, seed_matrix.cu:85, stays with the caller). */
typedef struct qm_depthmap qm_depthmap;

/* Depthmap(width, height, fx, cx, fy, cy, remap_1, remap_2, semi2dense_ratio),
 * depthmap.h:34-44 (note the fx, cx, fy, cy argument order). params NULL =
 * reference defaults.  device = CUDA ordinal. */
int qm_depthmap_create(qm_depthmap **out, int width, int height, float fx, float cx, float fy,
                       float cy, int semi2dense_ratio, const qm_params *params, int device);
int qm_depthmap_destroy(qm_depthmap *h);
/* Depthmap::add_frames(img_curr, T_curr_world), depthmap.h:46-47.
 * img: host u8 width x height, row pitch `stride` bytes.  T_curr_world:
 * world->camera.  *has_result = 1 when a new depth map is available (the
 * reference's boolean return). */
int qm_depthmap_add_frame(qm_depthmap *h, const uint8_t *img, size_t stride,
                          const float T_curr_world[12], int *has_result);
/* getDepthmap (depthmap.h:49): fused depth, -1 where invalid. stride in elements. */
int qm_depthmap_get_depth(qm_depthmap *h, float *out, size_t stride);
/* getDebugmap (depthmap.h:50): the sparse depth handed to the upsampler. */
int qm_depthmap_get_debug(qm_depthmap *h, float *out, size_t stride);
/* Fused variance sigma^2 per pixel of the last result (the fourth component
 * of the Bayesian seeds after fuse_currentmap, depth_fusion.cu:199-205); the
 * reference's Depthmap has no getter for it.  stride in elements. */
int qm_depthmap_get_variance(qm_depthmap *h, float *out, size_t stride);
/* getReferenceImage (depthmap.h:51): the image the last depth map belongs to. */
int qm_depthmap_get_reference(qm_depthmap *h, uint8_t *out, size_t stride);
/* getT_world_ref (depthmap.h:74). */
int qm_depthmap_get_T_world_ref(qm_depthmap *h, float T[12]);
/* 1 = run the semi-dense tracker on every frame (SeedMatrix::add_frames,
 * seed_matrix.cu:120-140): its projected depths seed the upsampler's sparse
 * input and appear in the debug map beside the BP node depths, as in the
 * reference.  0 (the default) = BP node depths only.  Only before the first
 * frame (QM_ERR_STATE after). */
int qm_depthmap_set_semidense(qm_depthmap *h, int enable);
/* Publisher::publishPointCloud (publisher.cpp:129-166) on the last result:
 * every pixel of the fused depth not below 0.1 gives the point
 * T_world_ref * (normalize(((x-cx)/fx, (y-cy)/fy, 1)) * depth) with the
 * reference image's intensity, in row-major pixel order, bit-identical to the
 * reference's host loop.  points: host, 4 floats (x, y, z, intensity) per
 * point; at most `capacity` points are written (width*height always
 * suffices); *count receives the number of points of the cloud. */
int qm_depthmap_get_point_cloud(qm_depthmap *h, float *points, size_t capacity, int *count);
/* getFx/Fy/Cx/Cy/Width/Height (depthmap.h:53-72). */
int qm_depthmap_get_camera(qm_depthmap *h, qm_camera *cam, int *width, int *height);

/* ------------------------------------------------------ batched streams
 * N independent Depthmap streams of uneven size on one device.  One
 * qm_batch_add_frames call runs the frame policy of every stream and then
 * the dense pipeline of all streams that produce a depth map, one kernel
 * launch per stage, replayed from a CUDA graph. */
typedef struct qm_batch qm_batch;
typedef struct qm_stream_desc {
  int width, height;
  qm_camera cam;
  int num_hyp;          /* 0 = params->num_hyp */
  int num_slots;        /* measurement slots (reference: 5) */
  int semi2dense_ratio; /* seed_matrix.cuh:51 */
} qm_stream_desc;

int qm_batch_create(qm_batch **out, int num_streams, const qm_stream_desc *descs,
                    const qm_params *params, int device);
int qm_batch_destroy(qm_batch *b);
/* imgs[i]: host u8 image of stream i (pitch strides[i] bytes), T_curr_world:
 * num_streams*12 floats, has_result: num_streams ints (out). */
int qm_batch_add_frames(qm_batch *b, const uint8_t *const *imgs, const size_t *strides,
                        const float *T_curr_world, int *has_result);
/* Pipelined form of qm_batch_add_frames: runs the frame policy of every
 * stream (has_result is final on return), enqueues the image uploads, the
 * dense pipeline and, for every stream i with a result and depth_outs[i] !=
 * NULL, the download of its fused depth into depth_outs[i] (row pitch
 * depth_strides[i] elements; NULL strides = dense rows), and returns
 * without waiting.  Up to two steps are in flight, so the uploads of one
 * step and the downloads of the previous one overlap the pipeline; host
 * buffers should be pinned for the copies to be asynchronous.  imgs may be
 * reused once the next qm_batch_submit or qm_batch_wait returns; depth_outs
 * are complete once qm_batch_wait returns (every other batch call also
 * waits first).  depth_outs may be NULL. */
int qm_batch_submit(qm_batch *b, const uint8_t *const *imgs, const size_t *strides,
                    const float *T_curr_world, int *has_result, float *const *depth_outs,
                    const size_t *depth_strides);
/* Waits for every submitted step. */
int qm_batch_wait(qm_batch *b);
int qm_batch_get_depth(qm_batch *b, int stream, float *out, size_t stride);
int qm_batch_get_debug(qm_batch *b, int stream, float *out, size_t stride);
int qm_batch_get_variance(qm_batch *b, int stream, float *out, size_t stride);
/* qm_depthmap_get_point_cloud for stream i of the batch. */
int qm_batch_get_point_cloud(qm_batch *b, int stream, float *points, size_t capacity,
                             int *count);
/* Fused depth of n streams in one call: streams[k] is written to outs[k]
 * (row pitch strides[k] elements); the downloads are issued together and
 * waited for once. */
int qm_batch_get_depths(qm_batch *b, int n, const int *streams, float *const *outs,
                        const size_t *strides);
/* Re-runs the dense pipeline of every stream on the frames already resident
 * on the device (no host transfers); used to time the device path alone. */
int qm_batch_run_resident(qm_batch *b);
/* Device pointer of stream i's fused depth map (row-major, dense). */
int qm_batch_device_depth(qm_batch *b, int stream, const float **dev_ptr);
/* 1 = replay captured CUDA graphs (default), 0 = launch stage by stage. */
int qm_batch_set_graphs(qm_batch *b, int enable);
/* qm_depthmap_set_semidense for every stream of the batch. */
int qm_batch_set_semidense(qm_batch *b, int enable);
/* k = 1..4 concurrent branches of the dense pipeline over consecutive
 * ranges of the streams that step together (the GPU fills one branch's
 * latency-bound stages -- coarse BP levels, line solves -- with the others'
 * work); 1 = one sequence over all of them; default 2.  Results do not
 * depend on it. */
int qm_batch_set_branches(qm_batch *b, int branches);
/* L2 budget, in bytes, of a job range of the belief propagation: each BP
 * level runs over consecutive streams whose level costs and messages fit in
 * it, so the range's half-sweeps hit L2.  0 = every level over all streams
 * at once (the default).  Results do not depend on it. */
int qm_batch_set_group_bytes(qm_batch *b, size_t bytes);
/* Coarse BP levels in one launch: the top pyramid levels with at most
 * max_cells cells in every stream (and at least two half-sweeps) run all
 * their half-sweeps in one launch, a cluster of blocks per stream with a
 * hardware cluster barrier between half-sweeps, instead of one launch per
 * half-sweep as the reference's bp_extract (bpextract.cu:122-143).  0 = one
 * launch per half-sweep everywhere; default 4096.  Results do not depend on
 * it. */
int qm_batch_set_coarse_bp(qm_batch *b, int max_cells);
/* 1 = with two or more branches, branch i + 1 starts once branch i's cost
 * volume is done, so the issue-bound cost kernel of one branch overlaps the
 * bandwidth-bound belief propagation of the previous one; 0 (the default,
 * measured faster) = all branches start together.  Results do not depend
 * on it. */
int qm_batch_set_stagger(qm_batch *b, int enable);
/* Launch shapes of the BP, line-solver and cost kernels: warps per block of
 * the BP half-sweeps and of the extraction (4, 8 or 16), rows per block of
 * the row solve (1, 2 or 4), columns per block of the column solve (2, 4 or
 * 8) and the cost kernel's register budget.  The reference fixes its block
 * shapes at compile time (bpextract.cu, depth_upsample.cu,
 * seed_matrix.cu launches); no counterpart. */
typedef struct qm_tune
{
  int sweep_warps, extract_warps, row_warps, col_lines;
  /* resident blocks per SM the cost kernel is built for (3, 4 or 5: the
   * register budget per thread, 80, 64 or 48; 0 in qm_batch_set_tune = the
   * default 5) */
  int cost_blocks;
} qm_tune;
/* 1 = autotune (the default): every set of streams that runs together times
 * three candidate shapes per kernel family on its first run (seven eager
 * runs that change no result) and keeps the fastest; 0 = the fixed shapes
 * (the defaults 8, 8, 2, 4, 5 unless qm_batch_set_tune set others).  Results
 * do not depend on the shapes. */
int qm_batch_set_autotune(qm_batch *b, int enable);
/* Fixes the shapes and turns autotune off.  QM_ERR_INVALID_ARG for a value
 * outside the sets above or a line-solver block whose lines exceed the
 * shared memory of a block for this batch's largest image. */
int qm_batch_set_tune(qm_batch *b, const qm_tune *t);
/* Shapes of the last dense-pipeline run (or profile). */
int qm_batch_get_tune(qm_batch *b, qm_tune *t);
/* Kernels launched by the last dense-pipeline run. */
int qm_batch_last_launches(qm_batch *b, int *count);
/* The cudaStream_t (as void*) every kernel of this batch is launched on;
 * record timing events on it. */
int qm_batch_stream(qm_batch *b, void **stream);
/* Kernel kinds reported by qm_batch_profile, in this order. */
#define QM_NUM_KERNEL_KINDS 11
/* quadtree, cost, pyramid, message init/upsample, bp half-sweep, extraction,
 * row solve, column solve, fuse transform, hole fill, fuse update.  The
 * message-init kind launches only at levels with fewer than two half-sweeps
 * (otherwise the half-sweeps write the inherited messages), and the hole-fill
 * kind reports 0 launches: hole filling runs inside the fuse update.  Runs
 * the resident pipeline once with eager launches, each
 * bracketed by CUDA events; ms[k] and launches[k] receive the summed device
 * time and the launch count of kind k.  No counterpart in the reference
 * (its printf timers measure CPU clock time, seed_matrix.cu:482-546). */
int qm_batch_profile(qm_batch *b, float ms[QM_NUM_KERNEL_KINDS],
                     int launches[QM_NUM_KERNEL_KINDS]);

/* ------------------------------------------- stage entry points --------
 * One keyframe, device buffers, asynchronous on `stream`.  Stages that need
 * scratch take a caller workspace whose size the *_workspace_size query
 * returns (no allocation inside). */

/* quadtree_image_kernal (quadtree.cu:17-77) as launched by
 * SeedMatrix::extract_depth (seed_matrix.cu:469-480).
 * levels: device u8 width*height (dense). */
int qm_quadtree(const uint8_t *img, size_t img_pitch, int width, int height,
                const qm_params *p, uint8_t *levels, void *stream);

/* image_to_cost + normalize_the_cost (depth_extract.cu:135-244; launch
 * seed_matrix.cu:486-524).  slots: HOST array of num_slots device image
 * pointers (pitch slot_pitch bytes); T_slot_ref: HOST num_slots*12 floats
 * (T_slot<-ref, the reference's FrameElement::transform).  Duplicated slots
 * are allowed (the reference's slot->ring map repeats frame 0, see
 * depth_extract.cu:153-166).  cost: device float (height/4)*(width/4)*num_hyp,
 * cell-major with hypotheses contiguous (the PIXEL_COST layout,
 * pixel_cost.cuh:11-37). */
int qm_cost_volume(const uint8_t *ref, size_t ref_pitch, int width, int height,
                   const qm_camera *cam, const uint8_t *levels, int num_slots,
                   const uint8_t *const *slots, size_t slot_pitch, const float *T_slot_ref,
                   const qm_params *p, float *cost, void *stream);

/* bp_extract (bpextract.cu:37-167) with cost_distribute, upsample, bp and
 * depth_extract (bpextract.cu:169-395).  cost: level-0 data from
 * qm_cost_volume (read only).  sparse: device f32 width*height; the pixel
 * (4x, 4y) of every quadtree-node cell receives its depth, all other pixels
 * are left as they are (the reference writes into debug_image,
 * seed_matrix.cu:530).  labels: device int32 (height/4)*(width/4) winning
 * hypothesis per cell, -1 where the cell is not a node origin (NULL to
 * skip).  messages: device f32 4*(height/4)*(width/4)*num_hyp final level-0
 * messages in the order up, down, left, right (NULL to skip).  cost,
 * messages and workspace must be 16-byte aligned (cudaMalloc'd memory is). */
int qm_bp_workspace_size(int width, int height, const qm_params *p, size_t *bytes);
int qm_bp_extract(const float *cost, int width, int height, const uint8_t *levels,
                  const qm_params *p, float *sparse, int32_t *labels, float *messages,
                  void *workspace, size_t workspace_bytes, void *stream);

/* global_upsample (depth_upsample.cu:20-57) with build_weight_row/col,
 * smooth_row and smooth_col (depth_upsample.cu:58-302).  dense: device f32
 * width*height.  Needs width % 16 == 0 and height % 8 == 0 (the reference
 * leaves the tails unwritten, depth_upsample.cu:111,216). */
int qm_upsample_workspace_size(int width, int height, size_t *bytes);
int qm_upsample(const float *sparse, const uint8_t *img, size_t img_pitch, int width, int height,
                const qm_params *p, float *dense, void *workspace, size_t workspace_bytes,
                void *stream);

/* qm_upsample without a workspace argument: no counterpart in the reference
 * (whose global_upsample cudaMallocs its buffers on every call).  For hosts
 * that cannot allocate device memory per call (a plugin host without a CUDA
 * allocator, a real-time loop that must not cudaMalloc after start-up).  It
 * allocates nothing: the row-pass scratch is a fixed device array of this
 * library of QM_UPSAMPLE_NOALLOC_MAX_PIXELS pixels (8 bytes each); larger
 * images return QM_ERR_INVALID_ARG.  The first call on a device sets up that
 * device (make it before any stream capture); so does the first call under
 * a different CUDA context (after cudaDeviceReset, or a context the host
 * made current itself), since the array's address is per context.  All calls on a device share
 * the scratch: calls that can overlap on the device race and give undefined
 * output, so issue them in order (e.g. on one stream).  Same limits as
 * qm_upsample otherwise. */
#define QM_UPSAMPLE_NOALLOC_MAX_PIXELS (1u << 20)
int qm_upsample_noalloc(const float *sparse, const uint8_t *img, size_t img_pitch, int width,
                        int height, const qm_params *p, float *dense, void *stream);

/* fuse_transform, hole_filling and fuse_currentmap (depth_fusion.cu:48-213;
 * launch seed_matrix.cu:553-597).  depth: device f32 width*height, in:
 * upsampled depth, out: fused depth (mu' or -1).  seeds_in / seeds_out:
 * device float4 (a, b, mu, sigma^2) per pixel (seeds_in is rewritten with
 * the transformed seeds, as the reference does).  T_income_last: HOST 12
 * floats.  table: device int32 width*height (out: source pixel index per
 * pixel, 0 = none). */
int qm_fuse_workspace_size(int width, int height, size_t *bytes);
int qm_fuse(float *depth, float *seeds_in, float *seeds_out, const float T_income_last[12],
            const qm_camera *cam, int width, int height, const qm_params *p, int32_t *table,
            void *workspace, size_t workspace_bytes, void *stream);

/* The point cloud of qm_depthmap_get_point_cloud for any depth map on the
 * device: depth (f32, row stride depth_stride floats), ref (u8, row pitch
 * ref_pitch bytes), T_world_ref HOST 12 floats.  points: device, 4 floats
 * per point, room for width*height points; count: device int, written when
 * the work on `stream` completes.  Workspace from
 * qm_point_cloud_workspace_size. */
int qm_point_cloud_workspace_size(int width, int height, size_t *bytes);
int qm_point_cloud(const float *depth, size_t depth_stride, const uint8_t *ref, size_t ref_pitch,
                   int width, int height, const qm_camera *cam, const float T_world_ref[12],
                   float *points, int *count, void *workspace, size_t workspace_bytes,
                   void *stream);

/* ------------------------------------------------ semi-dense tracker ----
 * The reference's LSD-style keyframe seeds (lsd_semidense.cu, seed_init.cu;
 * host sequence seed_matrix.cu:106-146,211-446) whose projection into the
 * incoming frame is the sparse depth the upsampler starts from.  Where the
 * reference's kernels race (in-place regularisation and hole filling,
 * propagation by atomicCAS with five retries, last-writer-wins projection)
 * this library is deterministic: neighbourhood passes read the state before
 * the pass, a propagation collision keeps the largest inverse depth and a
 * projection collision the smallest depth. */
#define QM_SD_INIT 1   /* first frame: seeds from the incoming image */
#define QM_SD_UPDATE 2 /* update_keyframe: stereo update, hole filling,
                          regularisation, projection */
#define QM_SD_SWITCH 3 /* update, then create_new_keyframe: propagation into
                          the incoming frame, which becomes the keyframe */
/* One step on device buffers.  key / inc: u8 width x height (dense rows), the
 * keyframe and the incoming frame (key unused for QM_SD_INIT).
 * T_income_key: HOST 12 floats, the keyframe-to-incoming transform
 * (income_transform * keyframe_transform.inv()).  trk / dep: device float4
 * per pixel, in and out: (valid > 0, blacklist, validity counter, 0) and
 * (idepth, variance, smooth idepth, smooth variance); zero-filled before the
 * first step.  debug: device f32 per pixel, out: the projected depths of the
 * confident seeds in the incoming frame, 0 elsewhere.  arith: QM_ARITH_*
 * (reference: the texture unit samples the images, as in the reference
 * kernels; IEEE: software bilinear with 8-bit weights, bit-exact with the
 * CPU oracle).  In reference arithmetic the call waits for the stream (its
 * texture objects live for the call). */
int qm_semidense_workspace_size(int width, int height, size_t *bytes);
int qm_semidense_step(const uint8_t *key, const uint8_t *inc, int width, int height,
                      const qm_camera *cam, const float T_income_key[12], int mode, int arith,
                      float *trk, float *dep, float *debug, void *workspace,
                      size_t workspace_bytes, void *stream);

/* ------------------------------------------------- differentiable path ----
 * For fitting the BP penalties (P1, P2) and per-pixel upsampling weight
 * factors to ground-truth depth.  No counterpart in the reference: it is the
 * training-side use of the stages above (the plain path keeps the hard
 * argmin).  Device pointers, asynchronous on `stream`.
 *
 * Soft BP: the hierarchical BP of qm_bp_extract followed by a softened
 * readout at the node cells: p(d) = softmax(-belief(d) / tau), depth =
 * 1 / (inv_depth_step * sum p(d) d + min_inv_depth), written at (4x, 4y) of
 * every node cell of `sparse` (zero elsewhere).  qm_bp_soft_backward takes
 * the same inputs, the workspace as the forward left it, and dL/d sparse,
 * and writes dL/dP1, dL/dP2 to grad_penalties (2 device doubles); it
 * recomputes the messages of each level instead of storing all of them.
 * cost and workspace 16-byte aligned. */
int qm_bp_soft_workspace_size(int width, int height, const qm_params *p, size_t *bytes);
int qm_bp_soft_forward(const float *cost, int width, int height, const uint8_t *levels,
                       const qm_params *p, float tau, float *sparse, void *workspace,
                       size_t workspace_bytes, void *stream);
int qm_bp_soft_backward(const float *cost, int width, int height, const uint8_t *levels,
                        const qm_params *p, float tau, const float *grad_sparse,
                        double *grad_penalties, void *workspace, size_t workspace_bytes,
                        void *stream);
/* The soft BP of qm_bp_soft_* in FP64 throughout (data terms, messages, the
 * readout and the adjoint), for checking gradients against FP64 finite
 * differences; the FP32 entry points above are the fitting path.  Same
 * arguments; the workspace (qm_bp_soft64_workspace_size) is its own. */
int qm_bp_soft64_workspace_size(int width, int height, const qm_params *p, size_t *bytes);
int qm_bp_soft64_forward(const float *cost, int width, int height, const uint8_t *levels,
                         const qm_params *p, float tau, float *sparse, void *workspace,
                         size_t workspace_bytes, void *stream);
int qm_bp_soft64_backward(const float *cost, int width, int height, const uint8_t *levels,
                          const qm_params *p, float tau, const float *grad_sparse,
                          double *grad_penalties, void *workspace, size_t workspace_bytes,
                          void *stream);
/* Upsampling with a weight factor per pixel: the systems of qm_upsample with
 * every inner edge weight (between a pixel and its left or upper neighbour)
 * multiplied by omega at that pixel, solved per line in FP64.  The backward
 * takes the forward's workspace unchanged and writes dL/d sparse and
 * dL/d omega.  width % 16 == 0, height % 8 == 0. */
int qm_upsample_w_workspace_size(int width, int height, size_t *bytes);
int qm_upsample_w_forward(const float *sparse, const uint8_t *img, size_t img_pitch, int width,
                          int height, const qm_params *p, const float *omega, float *dense,
                          void *workspace, size_t workspace_bytes, void *stream);
int qm_upsample_w_backward(const uint8_t *img, size_t img_pitch, int width, int height,
                           const qm_params *p, const float *omega, const float *grad_dense,
                           float *grad_sparse, float *grad_omega, void *workspace,
                           size_t workspace_bytes, void *stream);
/* Adjoint of the fusion update (fuse_currentmap) with respect to the
 * upsampled depth: depth_in = the depth qm_fuse was given, seeds_in = the
 * seeds as qm_fuse left them (transformed), table = its table. */
int qm_fuse_backward(const float *depth_in, const float *seeds_in, const int32_t *table,
                     int width, int height, const float *grad_fused, float *grad_depth,
                     void *stream);

#ifdef __cplusplus
}
#endif

#endif /* QM_CAPI_H */
