/* C ABI of the learned kerma denoiser's kernels (libccunet.so).
 *
 * The reference has no learned part; these entry points implement the 3D
 * U-Net denoiser that the engine's own Monte Carlo trains and against which
 * plain Monte Carlo measures the error.  Tensors are device pointers (16-byte aligned),
 * channels-last BF16 [B, D, H, W, C] activations with C a multiple of 16,
 * FP32 master weights and gradients.  Every call is asynchronous on the
 * given CUDA stream (NULL = legacy default stream) and returns 0 or a
 * negative CCU_E_* code with a message in ccu_last_error().
 */
#ifndef CHATCARLO_B200_UNET_H
#define CHATCARLO_B200_UNET_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CCU_VERSION 1

#define CCU_OK          0
#define CCU_E_INVALID (-1)   /* bad sizes, pointers or alignment */
#define CCU_E_DEVICE  (-6)   /* CUDA runtime failure */

int ccu_version(void);
const char* ccu_last_error(void);

/* Status bits set by the kernels (bit 0: a bounded tensor-core wait ran
 * out); reset clears them. */
int ccu_status(unsigned* status, int reset);

/* 3x3x3 "same" convolution on the tensor cores (tcgen05, BF16 in, FP32
 * accumulation).  The input is a [B, d, h, w, ca] concatenated on channels
 * with b [B, d/2, h/2, w/2, cb] read nearest-upsampled (b NULL, cb 0 for a
 * plain input).  weight: BF16 weights of 27 taps x cout x (ca + cb)
 * (tap = (dz+1)*9 + (dy+1)*3 + dx+1) in the packed order that
 * ccu_pack_weights writes (ccu_packed_weight_elems(cout, ca + cb)
 * elements); bias [cout] FP32 or NULL; relu 0/1.  Output channels [0, split)
 * go to out0 [.., split], multiplied by (mask0 > 0) when mask0 (same layout
 * as out0) is given; channels [split, cout) go to out1 [.., cout - split].
 * cout is one of 16, 32, 48, 64, 96, 128, 192; B*d*h*w < 2^31. */
int ccu_conv3d(const void* a, int ca, const void* b, int cb, int batch, int d, int h, int w, const void* weight,
               const float* bias, int cout, int relu, void* out0, int split, const void* mask0, void* out1,
               void* stream);

/* The network's last convolution and its 1 x 1 x 1 head in one pass: a
 * ReLU convolution of a [v][ca] (no second input) to 16 channels, and
 * out[v] = xlog[v] + head[16] + sum_j head[j] * bf16(act_j) -- the values
 * ccu_conv3d followed by ccu_head would give.  With the plane-stationary
 * kernel (path 0, weights in one pass) the head runs in its epilogue and the
 * activations are stored to act only when store_act is set; otherwise the
 * two calls are made, which needs act. */
int ccu_conv3d_head(const void* a, int ca, int batch, int d, int h, int w, const void* weight, const float* bias,
                    const float* head, const float* xlog, float* out, void* act, int store_act, void* stream);

/* Weight gradient of ccu_conv3d: dw[27][cout][ca + cb] (FP32) +=
 * sum over voxels of dz[v][co] * input[v + tap][ci].  The voxels are split
 * into `slices` ranges reduced with atomics.  cout in {16, 32, 64, 128}.
 * With w % 8 == 0 and ca, cb each 16, 32 or a multiple of 64 the input is
 * read by tensor-memory-accelerator tile loads (a second input is first
 * upsampled into a per-device buffer that the first such call allocates,
 * synchronously, and the process keeps), otherwise by the gathering kernel
 * (ccu_set_wgrad_path). */
int ccu_conv3d_wgrad(const void* a, int ca, const void* b, int cb, int batch, int d, int h, int w, const void* dz,
                     int cout, float* dw, int slices, void* stream);

/* db[c] += sum over voxels of dz[v][c]; c divides 256. */
int ccu_bias_grad(const void* dz, long long n_vox, int c, float* db, void* stream);

/* 2x2x2 average pooling, [B, d, h, w, c] -> [B, d/2, h/2, w/2, c]. */
int ccu_avgpool(const void* x, int batch, int d, int h, int w, int c, void* y, void* stream);

/* Backward of the pooling into a ReLU output x_act (full resolution):
 * dz_x += (x_act > 0) * gy[parent] / 8. */
int ccu_pool_backward(const void* gy, const void* x_act, int batch, int d, int h, int w, int c, void* dz_x,
                      void* stream);

/* Backward of the nearest upsampling of a ReLU output coarse_act:
 * dz_coarse = (coarse_act > 0) * sum over the 8 children of g_full
 * (d, h, w are the full-resolution sizes). */
int ccu_up_reduce(const void* g_full, const void* coarse_act, int batch, int d, int h, int w, int c, void* dz_coarse,
                  void* stream);

/* Output head (1x1x1 convolution 16 -> 1 with the input log kerma as
 * residual) and the weighted squared-error loss, head = 16 weights then the
 * bias:
 *   out[v] = xlog[v] + head[0:16] . d0[v] + head[16]
 *   loss = sum wgt (out - target)^2 * inv_wsum   (wgt NULL: all ones)
 * target, out, dz, dhead and loss may be NULL (inference).  With dz, also
 * the backward: dz[v] = (d0 > 0) * dloss/dout * head[0:16];
 * dhead[0..16] += dloss/dhead; loss[0] += loss. */
int ccu_head(const void* d0, const float* xlog, const float* target, const float* weight, const float* head,
             float inv_wsum, long long n_vox, float* out, void* dz, float* dhead, float* loss, void* stream);

/* Network input [n_vox, 16] BF16: normalised log kerma, density,
 * material one-hot (mat < n_mat <= 13), zeros, and in channel 15 unc[v]
 * (the input map's relative standard error, clipped by the caller) when
 * unc is not NULL. */
int ccu_input(const float* xlog, const float* density, const uint8_t* mat, int n_mat, const float* unc,
              long long n_vox, void* x, void* stream);

/* One Adam step (bias-corrected, decoupled weight decay wd) on n FP32
 * parameters; step counts from 1. */
int ccu_adam(float* p, const float* g, float* m, float* v, long long n, float lr, float b1, float b2, float eps,
             int step, float wd, void* stream);

/* ccu_adam on the gradient scaled by adaptive global-norm clipping: its
 * norm is capped at clip_ratio (>= 1) x the running mean of the capped
 * norms.  clip_state holds 3 doubles [sum of squares, running mean, last
 * scale]; zero them before the first step of a training run. */
int ccu_adam_clipped(float* p, const float* g, float* m, float* v, long long n, float lr, float b1, float b2,
                     float eps, int step, float wd, double* clip_state, float clip_ratio, void* stream);

/* Elements of a packed weight array for n output and c input channels
 * (both multiples of 16): 64 x n x ceil(27 c / 64); negative on error. */
long long ccu_packed_weight_elems(int n, int c);

/* BF16 weights of a layer from its FP32 master copy w32[27][cout][cin],
 * packed for ccu_conv3d: w for the forward convolution (n = cout, c = cin)
 * and, when wt is not NULL, wt for the backward-data convolution (n = cin,
 * c = cout; taps flipped, channels transposed). */
int ccu_pack_weights(const float* w32, int cout, int cin, void* w, void* wt, void* stream);

/* Which convolution kernel ccu_conv3d uses: 0 (default) the
 * plane-stationary kernel for 16 or 32 output channels (in channel passes
 * with an FP32 partial sum when the weights do not fit shared memory at
 * once; the partial lives in a per-device workspace of n_vox x cout x 4
 * bytes that the first such call allocates and the process keeps), else the
 * persistent halo kernel that streams z-planes through a shared-memory ring
 * where it applies (input and output channels <= 48), else the gathering
 * kernel; 1 always the gathering kernel; 2 the one-tile halo kernel where
 * it applies (channels <= 48, h % 16 == 0, w % 8 == 0; for comparisons);
 * 3 the streaming kernel with warp roles (loader, MMA and epilogue warps
 * handing off through mbarriers) where the streaming kernel applies; 4
 * path 0 without the plane-stationary kernel.  Process-wide. */
int ccu_set_conv_path(int path);

/* Kernel of ccu_conv3d_wgrad: 0 (default) tile loads where they apply, else
 * the gathering kernel; 1 the gathering kernel always.  Process-wide. */
int ccu_set_wgrad_path(int path);

/* Ring depth (input planes held in shared memory) of path 3: 0 (default)
 * chosen per layer to keep the most planes in flight per SM, else 4 .. 12
 * (a ring that does not fit a layer's shared memory makes ccu_conv3d fail
 * with CCU_E_INVALID).  Process-wide. */
int ccu_set_conv_ring(int ring);

/* Issue group of the plane-stationary kernel (path 0, 16 or 32 output
 * channels): 0 (default) chosen per layer, else 1 .. 3 input planes whose
 * MMA chains one thread interleaves (more independent accumulators in
 * flight, fewer CTAs per SM), reduced per layer to the largest group whose
 * tensor-memory regions fit 512 columns (3 for 16 output channels, 1 for
 * 32).  Process-wide. */
int ccu_set_conv_group(int group);

/* cudaMemsetAsync(p, 0, bytes) on the stream (gradient buffers). */
int ccu_zero(void* p, long long bytes, void* stream);

/* Test GEMM of the tensor-core path: d[m][n] (FP32) = a . b^T with a
 * [m][k] (a_mn = 0) or [k][m] (a_mn = 1) and b [n][k] (b_mn = 0) or
 * [k][n] (b_mn = 1), BF16; m % 128 == 0, n % 16 == 0 with n <= 256,
 * k % 64 == 0. */
int ccu_gemm_test(const void* a, const void* b, float* d, int m, int n, int k, int a_mn, int b_mn, void* stream);

#ifdef __cplusplus
}
#endif

#endif
