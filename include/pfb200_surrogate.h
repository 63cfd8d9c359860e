/* pfb200_surrogate.h -- learned relaxation surrogate of the 2D update.
 *
 * No counterpart in the reference: the reference relaxes every system with
 * the explicit Euler step only. This interface adds (1) 3x3 "same"
 * convolutions on bfloat16 activations with binary32 accumulation on the
 * tcgen05 tensor cores (forward, data gradient, weight gradient), (2) a small
 * U-Net built from them that maps a 64 x 64 crop around one cell (its phi and
 * the sum of the other cells' phi^2) to the cell's phi after a fixed number of
 * passive relaxation steps, with its training step, and (3) the jump of a
 * pfb_sim2d system by that network, after which the plain step resumes and
 * judges the result by its residual.
 *
 * Activation layout ("padded NHWC"): image b of H x W pixels and C channels
 * occupies (H + 2) * (W + 2) * C bfloat16 values, position
 * q = (y + 1) * (W + 2) + (x + 1) for pixel (y, x), channels innermost, with a
 * zero border one pixel wide. Kernels never write the top and bottom border
 * rows, so buffers start zeroed. All buffers 16-byte aligned.
 *
 * Return values: PFB_OK (0) or a negative PFB_E_* code (pfb200.h), with the
 * text in pfb_last_error(). */
#ifndef PFB200_SURROGATE_H
#define PFB200_SURROGATE_H

#include <stddef.h>
#include <stdint.h>

#include "pfb200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- convolutions ---------------------------------------------------------- */

/* out = conv3x3(x, W) (+ bias[co]) (ReLU if relu) (* (gate > 0) if gate),
 * computed for `batch` images of H x W; x has cin channels, the output cout.
 * y receives bfloat16 (round to nearest), y_f32 binary32; either may be null
 * but not both. w_packed comes from pfb_conv3x3_pack. Built channel pairs
 * (cin, cout): (16, 16), (16, 32), (32, 16), (32, 32). The border columns of
 * the output rows are written as zero. */
int pfb_conv3x3_forward(const void* x, void* y, float* y_f32, const void* w_packed,
                        const float* bias, const void* gate, int batch, int H, int W, int cin,
                        int cout, int relu, void* stream);

/* Pack binary32 weights w_oihw[cout][cin][3][3] into the bfloat16 operand
 * layout of pfb_conv3x3_forward (9 * cin * cout values). transpose != 0 packs
 * the flipped, transposed weights of the data gradient: running
 * pfb_conv3x3_forward with them on dY (cout channels) gives dX (cin
 * channels). */
int pfb_conv3x3_pack(const float* w_oihw, void* w_packed, int cin, int cout, int transpose,
                     void* stream);

/* Bytes of the workspace pfb_conv3x3_wgrad needs for these sizes: binary32
 * partial sums, one block per CTA, added afterwards in a fixed order. */
size_t pfb_conv3x3_wgrad_workspace(int batch, int H, int W, int cx, int cy);

/* dw_oihw[cy][cx][3][3] = sum over images and pixels of dY[q][co] *
 * x[q + tap][ci], and db[co] = sum dY[q][co] (db may be null); x has cx
 * channels, dy cy (its border must be zero). Overwrites dw and db.
 * Deterministic. Built pairs (cx, cy) as for the forward pass. */
int pfb_conv3x3_wgrad(const void* x, const void* dy, float* workspace, size_t workspace_bytes,
                      float* dw_oihw, float* db, int batch, int H, int W, int cx, int cy,
                      void* stream);

/* pfb_conv3x3_wgrad without a caller workspace. No counterpart in the
 * reference. For callers that cannot allocate device memory for this
 * library: hosts whose device memory belongs to their own pool allocator (a
 * training framework's caching allocator, a serving engine's preallocated
 * arena) and that forbid a raw cudaMalloc, which would take memory outside
 * their budget and, being synchronizing, stall their streams. The partial
 * sums live in a fixed 4 MiB array of the library that every GPU loading it
 * holds until exit; sizes needing more (pfb_conv3x3_wgrad_workspace above
 * 4 MiB, e.g. more than 56 images of 64 x 64 with 32 -> 32 channels) are
 * rejected with PFB_E_ARG. Nothing in the array has to start at zero (each
 * call overwrites what it reads; a CTA whose bounded MMA wait gave up writes
 * NaN, so such a result is NaN, never stale data, and pfb_conv_status bit 0
 * is set). The first call on a device looks up the array's device address
 * with that device current and keeps it for the process; make that first
 * call before any stream capture, and do not call it after a
 * cudaDeviceReset of that device (the kept address would be stale). Calls
 * that overlap on the GPU share the array and race: serialise them.
 * Allocates nothing; same results as pfb_conv3x3_wgrad. */
int pfb_conv3x3_wgrad_noalloc(const void* x, const void* dy, float* dw_oihw, float* db,
                              int batch, int H, int W, int cx, int cy, void* stream);

/* Sticky device status of the convolution kernels: bit 0 = a wait for the
 * tensor-core MMAs gave up (the kernel skipped its output). clear != 0
 * resets it. */
int pfb_conv_status(unsigned* out, int clear);
/* (pfb_conv_status bit 1: the persistent forward found its shared memory
 * misaligned for TMA and computed nothing.) */
/* Forward / data-gradient kernel choice. 2: every built channel pair runs as
 * a persistent warp-specialised kernel (TMA loads of the activation tiles
 * into a two-stage ring, tcgen05 MMAs into two TMEM accumulators, epilogue
 * warps draining the previous tile) where the image width allows one TMA box
 * per half tile (W <= 124); 1 (default): the persistent kernel for the
 * 32 -> 32 pair only, the one where it is faster (124 vs 134 us at 512 x 64^2
 * on a B200; 7-27 % slower at 16 -> 32, 32 -> 16 and 16 -> 16); 0: one CTA per
 * tile that stages, multiplies and writes in turn. All give the same values.
 * PFB_E_ARG for any other mode. */
int pfb_conv_set_pipeline(int mode);

/* ---- relaxation measurements and crops of a pfb_sim2d system ---------------
 * (binary32 pools only; PFB_E_CONFIG otherwise) */

/* Advance `s` by one step and measure that step's residual over every cell:
 * linf = max |phi_n^{k+1} - phi_n^k| / dt over the lattice sites of the
 * cell's old and new windows (world coordinates), rms = the root mean square
 * of the same quantity over those sites. Either output may be null. */
int pfb_sim2d_residual_step(pfb_sim2d* s, double* linf, double* rms);

/* Network input of every cell of `s` (num_cells padded 66 x 66 images of 16
 * bfloat16 channels: phi_n and the sum over the other cells of
 * min(phi_m^2, 4), on the 64 x 64 lattice crop centred at the cell's
 * rounded centroid; channel 2 zero), the binary32 phi_n crops (num_cells x
 * 64 x 64, may be null) and the crop origins (num_cells x 2 ints, x then
 * y). Device buffers; runs on the system's stream. */
int pfb_sur2d_extract(pfb_sim2d* s, void* x0, float* phi_crop, int* origins);

/* As pfb_sur2d_extract on crops at the given origins, with channel 2 =
 * (phi_n - prev) * hist_scale when prev (num_cells x 64 x 64 crops of an
 * earlier step at the same origins) is not null: the recent rate of change
 * when hist_scale = 1 / (steps between them x dt). */
int pfb_sur2d_extract_at(pfb_sim2d* s, const int* origins, const float* prev, float hist_scale,
                         void* x0, float* phi_crop);

/* out = phi_n on the 64 x 64 crops at `origins` (binary32), minus `minus`
 * when it is not null (e.g. the crops of an earlier step: the increment). */
int pfb_sur2d_crop_phi(pfb_sim2d* s, const int* origins, const float* minus, float* out);

/* phi_n += dphi (num_cells x 64 x 64) at the crop sites inside each cell's
 * window, then the cells' moments and the current aggregate are rebuilt from
 * the edited field. */
int pfb_sur2d_insert(pfb_sim2d* s, const int* origins, const float* dphi);

/* ---- the surrogate network -------------------------------------------------
 * Input channels: phi_n, the others' sum of phi^2, phi_n's recent rate.
 * A U-Net of eight 3x3 convolutions of width 32 (ReLU; 2x2 average pool and
 * nearest upsampling with a skip connection between 64^2 and 32^2) mapping a
 * crop from pfb_sur2d_extract to the increment of phi_n over the relaxation
 * interval it was trained on. bfloat16 activations, binary32 accumulation,
 * master weights, gradients and Adam moments. */
typedef struct pfb_sur2d pfb_sur2d;

/* Buffers for batches of up to max_batch crops; weights He-normal from
 * `seed` (the last layer zero: the untrained network predicts no change). */
pfb_sur2d* pfb_sur2d_create(int max_batch, unsigned long long seed, int device);
void pfb_sur2d_destroy(pfb_sur2d* n);
/* Number of binary32 parameters (weights [cout][cin][3][3] then bias, per
 * layer in order; padded channels included). */
long long pfb_sur2d_num_params(const pfb_sur2d* n);
int pfb_sur2d_get_params(pfb_sur2d* n, float* out);     /* host buffer */
int pfb_sur2d_set_params(pfb_sur2d* n, const float* in); /* resets Adam */
int pfb_sur2d_get_grads(pfb_sur2d* n, float* out);      /* host buffer */

/* dphi (batch x 64 x 64, binary32) = network(x0) for `batch` device crops. */
int pfb_sur2d_predict(pfb_sur2d* n, const void* x0, float* dphi, int batch);

/* Gather crops idx[0..batch) of a device training set (x_all: inputs as
 * pfb_sur2d_extract writes them, t_all: target increments, 64 x 64 each),
 * compute the mean-squared error of channel 0 and every parameter's
 * gradient (no update). loss may be null (no host synchronisation). */
int pfb_sur2d_loss_grad(pfb_sur2d* n, const void* x_all, const float* t_all, const int* idx,
                        int batch, double* loss);
/* pfb_sur2d_loss_grad followed by one Adam step (beta 0.9, 0.999, eps 1e-8)
 * with learning rate lr. */
int pfb_sur2d_train_step(pfb_sur2d* n, const void* x_all, const float* t_all, const int* idx,
                         int batch, float lr, double* loss);
int pfb_sur2d_sync(pfb_sur2d* n);

/* Jump every cell of `s` by the network (extract, predict, insert, rebuild)
 * on the system's stream; returns after it completed. */
int pfb_sur2d_jump(pfb_sur2d* n, pfb_sim2d* s);
/* The same with the rate input: crops now, history_steps plain steps,
 * crops again with channel 2 = their difference * hist_scale, then the
 * jump. */
int pfb_sur2d_jump_history(pfb_sur2d* n, pfb_sim2d* s, int history_steps, float hist_scale);

/* Device milliseconds per forward pass over `batch` crops (CUDA events). */
int pfb_sur2d_bench_forward(pfb_sur2d* n, int batch, int iters, double* ms);

#ifdef __cplusplus
}
#endif

#endif /* PFB200_SURROGATE_H */
