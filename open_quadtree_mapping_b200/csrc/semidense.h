// Semi-dense tracker: per-stream job descriptor of one frame step and the
// batched launcher (k_semidense.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace qm
{

enum SdMode
{
  kSdNone = 0,   // stream not stepped this frame
  kSdInit = 1,   // first frame: seeds from the incoming image
  kSdUpdate = 2, // stereo update, hole filling, regularisation, projection
  kSdSwitch = 3  // update, then propagation into the new keyframe
};

// One stream's semi-dense step.  Images are W x H; the float images share
// the row pitch `pitch` (floats).  Seeds live in two buffers each of trk
// (valid, blacklist, validity counter, -) and dep (idepth, variance, smooth
// idepth, smooth variance); `cur` holds the state before and after the step.
struct SdJob
{
  int W, H;
  float fx, fy, cx, cy;
  int mode;                   // SdMode
  const uint8_t *inc;         // incoming frame, u8 dense
  float *inc_f;               // its float copy (written by the step)
  const float *key_f;         // the keyframe's float image
  size_t pitch;               // of inc_f and key_f, in floats
  cudaTextureObject_t inc_tex, key_tex; // linear-filtered views of them
  float4 *trk[2], *dep[2];
  int cur;
  float *debug;               // W x H projected depths (0 elsewhere)
  unsigned long long *zkey;   // W x H z-buffer, all ones between steps
  float T[12];                // T_income<-key
};

struct SdBatch
{
  const SdJob *jobs; // device (null: the single job `one`)
  const int *prefix; // device: block prefix over the jobs (njobs + 1)
  int njobs;
  SdJob one;
};

int sd_blocks(int W, int H);
// enqueues the whole step sequence; returns the number of launches
int launch_semidense(const SdBatch &B, int blocks, int ieee, cudaStream_t s);
// float copy of a u8 image (dense rows of W bytes) with row pitch `pitch`
// floats
void launch_u8_to_f32(const uint8_t *src, int W, int H, float *dst, size_t pitch,
                      cudaStream_t s);
// row pitch (floats) of a W-wide float image that a pitch-2D texture accepts
// on the current device
size_t sd_texture_pitch(int W);
// linear-filtered, clamp-addressed view of a float image (unnormalised
// coordinates), as the reference's bindTexture sets it up
cudaTextureObject_t sd_make_texture(const float *img, int W, int H, size_t pitch);

} // namespace qm
