// msg_conv_tc.cuh -- tensor-core (tcgen05 / TMEM / TMA) forward pass of the 16-channel
// 3x3x3 CNN of the learned initial guess, used for inference inside the time loop.
#pragma once
#include "msg_common.cuh"
#include "../../include/msg123_gpu.h"
#include <cuda_bf16.h>

namespace msg {

// Activations of one grid in the halo-padded, chunk-planar layout the kernel reads with TMA:
// element (chunk, z, y, x, c) at ((chunk * pz + z) * py + y) * px + x) * 8 + c, with
// px = nx + 2 (and so on), interior cell (ix, iy, iz) at (ix + 1, iy + 1, iz + 1),
// chunk = channel / 8, c = channel % 8.  The halo stays zero (the 3x3x3 zero padding).
struct ConvPlan;

// (Re)build the plan for an nx x ny x nz grid on the current device.
int conv_plan_get(ConvPlan **plan, int nx, int ny, int nz);
void conv_plan_free(ConvPlan *plan);
// Padded input buffer (features) of the plan; 2 * plane * 8 bf16.
__nv_bfloat16 *conv_plan_input(ConvPlan *plan);
size_t conv_plan_plane(ConvPlan *plan);
// Compact [N][16] bf16 features -> the plan's padded input buffer.
int conv_plan_load_compact(ConvPlan *plan, const __nv_bfloat16 *x, cudaStream_t s);

// Four convolutions (GELU after the first three) from the plan's input buffer.
// wpk: weights packed for the tensor cores by conv_pack_weights; bias: bias[l] points at
// 16 floats of layer l.  *out receives the output channel in interior order (N floats,
// owned by the plan).
// withhold >= 0 (tests only): the first layer never loads the first box of that segment, so the
// consumer's bounded wait runs out and the pass reports an error instead of hanging.
int conv_forward_tc(ConvPlan *plan, const __nv_bfloat16 *wpk, const float *const bias[4], cudaStream_t s,
                    const float **out, int withhold = -1);
// Synchronise the stream and report a wait that ran out inside the last forward pass.
int conv_check(ConvPlan *plan, cudaStream_t s);

// Pack W[tap][co][ci] (FP32 master weights, per-layer stride `layer_stride` floats) into
// the tensor-core layout of the z-march kernel: [layer][rotation][in-plane tap][k chunk]
// [48 columns][8 ci] bf16, conv_packed_elems() elements.
size_t conv_packed_elems();
int conv_pack_weights(const float *w32, int layer_stride, __nv_bfloat16 *wpk, cudaStream_t s);

}  // namespace msg
