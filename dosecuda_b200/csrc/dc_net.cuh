// dc_net.cuh — building blocks of the photon-dose surrogate network.
//
// Activations are bf16, channels-last (n, d, h, w, c) with c contiguous, so a
// voxel's channels form 16-byte chunks of 8 channels: the unit of every
// shared-memory tile and of every ldmatrix row.  Convolutions are implicit
// GEMMs on the tensor cores (mma.sync m16n8k16, bf16 operands, fp32
// accumulation):
//   * conv_gather: out[o] = sum_t W_t^T in[g(o, t)] — 3x3x3 stride-1 pad-1
//     (27 taps, same grid) or 2x2x2 stride-2 (8 taps, half grid);
//   * conv_up: out[2q + t] = W_t^T in[q] — 2x2x2 stride-2 transposed conv;
//   * conv_wgrad: G_t = sum_o P[g(o, t)] Q[o]^T — the weight gradient of
//     either gather form (and, with P/Q swapped, of conv_up).
// The backward-data pass of each form is the other form with repacked weights
// (flipped taps and/or transposed channel roles), so three kernels cover the
// forward and both backward passes of the whole encoder-decoder.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace dc {
namespace net {

using bf16 = __nv_bfloat16;

// Gather-convolution modes.
constexpr int kConv3 = 0;   // 3x3x3, stride 1, pad 1; output grid == input grid
constexpr int kDown2 = 1;   // 2x2x2, stride 2; output grid == input grid / 2

// Number of uint2 fragments of a packed weight set: ceil(T*K/16) k-steps x
// (N/8) n-tiles x 32 lanes.
long long packed_fragments(int taps, int k_per_tap, int n);

// Device for the following calls on this thread: each helper validates its
// arguments first and only then makes it current.
void set_call_device(int gpu_id);

// Enqueue helpers (throw dc::Error on bad arguments / launch failure).
void pack_weights(const float *master, int taps, int a, int b, int flip, int trans, uint2 *out,
                  cudaStream_t s);
void conv_gather(int mode, const bf16 *x, int n, int d, int h, int w, int cin, const uint2 *wpk,
                 long long wpk_frags, int cout, bf16 *y, double *stats, cudaStream_t s);
void conv_up(const bf16 *x, int n, int d, int h, int w, int cin, const uint2 *wpk, long long wpk_frags, int cout,
             const bf16 *addend, bf16 *y, cudaStream_t s);
void conv_wgrad(int mode, const bf16 *p, const bf16 *q, int n, int d, int h, int w, int ca, int cb, float *grad,
                cudaStream_t s);
void norm_finalize(const double *stats, int n, int c, long long count, const float *gamma, const float *beta,
                   float eps, float *coef, cudaStream_t s);
void norm_act(const bf16 *y, int n, long long vox, int c, const float *coef, float slope, bf16 *a, cudaStream_t s);
void norm_stats_act(const bf16 *y, int n, long long vox, int c, const double *stats, long long count,
                    const float *gamma, const float *beta, float eps, float slope, float *coef, bf16 *out,
                    cudaStream_t s);
void norm_act_bwd(const bf16 *y, const bf16 *da, int n, long long vox, int c, const float *coef,
                  const float *gamma, float slope, double *red, bf16 *dy, float *dgamma, float *dbeta,
                  cudaStream_t s);
void pack_input(const float *terma, const float *density, long long vox, float terma_scale, bf16 *x8,
                cudaStream_t s);
void head_fwd(const bf16 *g, long long vox, int c, const float *w, const float *bias, const float *mask,
              float mask_thr, float scale, float *out, cudaStream_t s);
void head_loss_bwd(const bf16 *g, long long vox, int c, const float *w, const float *pred, const float *target,
                   float inv_count, const float *inv_count_dev, double *loss, bf16 *dg, float *dw, float *dbias,
                   cudaStream_t s);

// Tensor-core (tcgen05) 3x3x3 convolution for grids of x extent 128
// (dc_net_tc.cu): weights prepacked by pack_weights_tc.
long long packed_tc_bytes(int cin, int cout);
void pack_weights_tc(const float *master, int taps, int a, int b, int flip, int trans, void *out, cudaStream_t s);
bool conv_tc_supported(int d, int h, int w, int cin, int cout);
void conv_tc(const bf16 *x, int n, int d, int h, int w, int cin, const void *wtc, long long wtc_bytes, int cout,
             bf16 *y, double *stats, cudaStream_t s);
int take_tc_error();
int tc_wait_selftest(cudaStream_t s);

}  // namespace net
}  // namespace dc
