/*
 * ptycho_b200.h -- C ABI of the B200 (sm_100a) far-field ptychography library.
 *
 * All entry points are stream-ordered and asynchronous: they enqueue work on
 * `stream` and return without synchronising.  The caller owns every buffer;
 * the library allocates nothing (scratch memory is a caller-provided
 * workspace whose size is returned by the matching *_workspace_size query).
 * Pointers are device pointers unless stated otherwise.  Complex arrays are
 * interleaved (re, im) float32 pairs ("complex64"), row-major.  No call
 * throws; each returns a ptycho_status.  Calls are reentrant; two calls that
 * share a workspace must be ordered on one stream.
 *
 * Reference interfaces replaced (paths relative to the reference tree):
 *   utils/optics.py:102-112   forward_imaging_model      -> ptycho_forward_intensity
 *   Recovery.py:288-307,316   per-frame loss + autograd  -> ptycho_fwd_adj
 *   utils/optics.py:68-99     scan_positions_to_pixels   -> ptycho_scan_to_pixels
 *   models/complex_inr.py:130-145,279,294  tcnn HashGrid Encoding
 *                                                   -> ptycho_hashgrid_{forward,backward}
 *   models/complex_inr.py:6-82,308-314     ComplexMLP.net
 *                                                   -> ptycho_cmlp_{forward,backward}
 *   Recovery.py:238-241,321   torch.optim.Adam.step      -> ptycho_adam_step
 */
#ifndef PTYCHO_B200_H
#define PTYCHO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* ptycho_stream_t; /* same type as cudaStream_t */

typedef enum {
  PTYCHO_OK = 0,
  PTYCHO_ERR_INVALID_ARG = 1,      /* null pointer, negative size, bad enum */
  PTYCHO_ERR_UNSUPPORTED_SIZE = 2, /* size outside what the entry point takes */
  PTYCHO_ERR_MISALIGNED = 3,       /* pointer not aligned as documented */
  PTYCHO_ERR_WORKSPACE = 4,        /* workspace too small */
  PTYCHO_ERR_LAUNCH = 5,           /* CUDA launch failed (see cudaGetLastError) */
  PTYCHO_ERR_WINDOW = 6,           /* (device flag) a scan window left the canvas */
  PTYCHO_ERR_TIMEOUT = 7           /* (device flag) a bounded wait gave up */
} ptycho_status;

typedef enum {
  PTYCHO_LOSS_SMOOTH_L1 = 0, /* Recovery.py:294-295  F.smooth_l1_loss, beta 1, mean */
  PTYCHO_LOSS_FD = 1,        /* Recovery.py:296-302  gradient-difference loss       */
  PTYCHO_LOSS_POISSON = 2,   /* Recovery.py:303-305  I - Imeas*log(I+1e-8), mean     */
  PTYCHO_LOSS_INTENSITY_GRAD = 3 /* `Imeas` holds an upstream gradient dL/dI: the call is
                                    the backward of ptycho_forward_intensity for any loss
                                    (loss_per_pattern = sum I*dL/dI)                     */
} ptycho_loss_type;

/* flags for ptycho_fwd_adj */
#define PTYCHO_FLAG_ACCUMULATE 1u /* add into dO/dP instead of overwriting */

/* Human-readable name of a status code (static string). */
const char* ptycho_status_string(int status);

/* Library version as major*10000 + minor*100 + patch. */
int ptycho_version(void);

/* ---------------------------------------------------------------------- *
 * Scan positions and batches.  The scan is described once for all F frames:
 *   tl    [F][2] int32  top-left window corner (tlY, tlX) of frame f
 *                       (utils/optics.py:91-92; bottom-right = tl + (M, N))
 *   Imeas [F][M][N] float32 measured intensities, frames first (the
 *                       reference keeps [M][N][F], Recovery.py:103-104,289)
 * A call processes a batch of B frame ids `batch` [B] int32 (the
 * reference's `perm[batch_start : batch_start + batch_size]`,
 * Recovery.py:244-249); `batch` may be NULL for frames 0..B-1 (B <= F).
 * A frame id outside [0, F) or a window outside the canvas is skipped: its
 * outputs are NaN / zero and PTYCHO_ERR_WINDOW is raised in `status_out`
 * (device int32, may be NULL; only ever set, never cleared).
 * ---------------------------------------------------------------------- */

/* ---------------------------------------------------------------------- *
 * Forward model.  Replaces utils/optics.py:102-112 forward_imaging_model,
 * batched: for b < B, with f = batch[b],
 *   I_out[b] = | fftshift( fft2( P * O[tlY_f : tlY_f+M, tlX_f : tlX_f+N] ) ) |^2
 * O [H][W] complex64, P [M][N] complex64, I_out [B][M][N] float32.
 * ptycho_forward_intensity takes M == N in {64, 128, 256} (the fused
 * kernels; 256: one 4-CTA thread-block cluster per pattern) and needs no
 * scratch memory; other shapes return PTYCHO_ERR_UNSUPPORTED_SIZE.
 * ptycho_forward_intensity_ws takes any 1 <= M, N <= 4096 (the reference
 * accepts any probe shape, Recovery.py:290): shapes the fused kernels do not
 * cover run as gather, mixed-radix row and column DFTs and an intensity
 * pass over a workspace of ptycho_forward_intensity_workspace_size(M, N, B)
 * bytes (256-byte aligned; the fused shapes need none).
 * ---------------------------------------------------------------------- */
int ptycho_forward_intensity(const float* O, int H, int W, const float* P, int M, int N,
                             const int32_t* tl, int F, const int32_t* batch, int B,
                             float* I_out, int32_t* status_out, ptycho_stream_t stream);

size_t ptycho_forward_intensity_workspace_size(int M, int N, int B);

int ptycho_forward_intensity_ws(const float* O, int H, int W, const float* P, int M, int N,
                                const int32_t* tl, int F, const int32_t* batch, int B, float* I_out,
                                void* workspace, size_t workspace_bytes, int32_t* status_out,
                                ptycho_stream_t stream);

/* ---------------------------------------------------------------------- *
 * Fused forward + loss + adjoint.  Replaces the per-frame loop of
 * Recovery.py:288-307 and the autograd backward of Recovery.py:316 for the
 * pixel terms: for the B frames of the batch it computes
 *   loss_per_pattern[b] = mean_pixels loss(I_b, Imeas_{batch[b]})   (FP64)
 *   loss_total[0]       = sum_b loss_per_pattern[b]                (FP64)
 *   dO = d loss_total / d O,  dP = d loss_total / d P
 * in torch's convention for complex leaves (dL/dRe + i dL/dIm).  Gradients
 * are summed in a fixed order (deterministic, no floating-point atomics).
 * loss_per_pattern (B doubles), loss_total (1 double), dO [H][W] and
 * dP [M][N] may each be NULL to skip that output; when dO and dP are both
 * NULL the adjoint is not computed.  With PTYCHO_FLAG_ACCUMULATE dO/dP are
 * added to instead of overwritten.  workspace: device scratch of at least
 * ptycho_fwd_adj_workspace_size() bytes, 256-byte aligned.  Imeas must be
 * 16-byte aligned (each pattern's measurement is fetched by a bulk copy).
 * Probes: M == N in {64, 128} run the fused kernels; M == N == 256 runs
 * three line-DFT kernels over the workspace (smooth-L1, Poisson and the
 * intensity-gradient code; batches of 192 or more also take dP from the
 * inverse-row kernel) or, for the FD loss, one 4-CTA cluster per pattern;
 * any other 1 <= M, N <= 4096 (non-square, odd, 96, 192, ...) runs the
 * general path: the same losses and gradients through workspace passes
 * (gather, row and column DFTs of any length, loss, inverse DFTs), then the
 * same assembly.
 * ---------------------------------------------------------------------- */
size_t ptycho_fwd_adj_workspace_size(int H, int W, int M, int N, int B);

int ptycho_fwd_adj(const float* O, int H, int W, const float* P, int M, int N,
                   const int32_t* tl, const float* Imeas, int F, const int32_t* batch, int B,
                   int loss_type, double* loss_per_pattern, double* loss_total, float* dO,
                   float* dP, unsigned flags, void* workspace, size_t workspace_bytes,
                   int32_t* status_out, ptycho_stream_t stream);

/* ---------------------------------------------------------------------- *
 * Multi-resolution hash encoding.  Replaces the tiny-cuda-nn
 * `tcnn.Encoding(n_input_dims=2, {"otype": "HashGrid", ...})` of
 * models/complex_inr.py:130-145 (called at :279, :294).  coords [N][2]
 * float32 in [0,1]; table [entries][2] float32 (entries =
 * ptycho_hashgrid_entries()); features [N][n_levels*2] float32.
 * Level l: scale s = base*per_level_scale^l - 1, r = ceil(s)+1 vertices per
 * axis, position x*s + 0.5, bilinear weights; dense index ix + iy*r when
 * r^2 (rounded up to a multiple of 8) fits in 2^log2_hashmap_size entries,
 * otherwise (ix ^ iy*2654435761) mod 2^log2_hashmap_size.  per_level_scale
 * is taken as float32 (as in a tiny-cuda-nn JSON config); scales are formed
 * from it in double precision and rounded to float32.
 * ---------------------------------------------------------------------- */
int ptycho_hashgrid_entries(int n_levels, int log2_hashmap_size, int base_resolution,
                            float per_level_scale);

int ptycho_hashgrid_forward(const float* coords, int N, const float* table, int n_levels,
                            int log2_hashmap_size, int base_resolution, float per_level_scale,
                            float* features, ptycho_stream_t stream);

/* The same encoding written feature-major: features_planar [n_levels*2][N]
 * (feature f of coordinate n at f*N + n).  One thread per (coordinate, level),
 * coalesced stores; values bitwise those of ptycho_hashgrid_forward. */
int ptycho_hashgrid_forward_planar(const float* coords, int N, const float* table, int n_levels,
                                   int log2_hashmap_size, int base_resolution, float per_level_scale,
                                   float* features_planar, ptycho_stream_t stream);

/* Static contributions of fixed coordinates: for each (coordinate n,
 * level l, corner k), index i = (n*n_levels + l)*4 + k: key[i] = table entry,
 * item[i] = n*n_levels + l (feature pair), weight[i] = bilinear weight.
 * Sort (key, item, weight) by key, stably, once; then pass the segment
 * starts of ptycho_hashgrid_segments to ptycho_hashgrid_backward. */
int ptycho_hashgrid_contrib(const float* coords, int N, int n_levels, int log2_hashmap_size,
                            int base_resolution, float per_level_scale, int32_t* key,
                            int32_t* item, float* weight, ptycho_stream_t stream);

/* start [n_entries + 1]: start[e] = first sorted position whose key >= e. */
int ptycho_hashgrid_segments(const int32_t* sorted_key, long long K, int n_entries,
                             int32_t* start, ptycho_stream_t stream);

/* dtable[e] (+)= sum over e's contributions, in sorted order, of
 * weight * dfeatures[item]: the table-gradient scatter as a deterministic
 * gather (no atomics). */
int ptycho_hashgrid_backward(const int32_t* start, const int32_t* item, const float* weight,
                             const float* dfeatures, int N, int n_levels, int log2_hashmap_size,
                             int base_resolution, float per_level_scale, float* dtable,
                             int accumulate, ptycho_stream_t stream);

/* The same backward for a feature gradient stored feature-major: dfeatures_planar
 * [n_levels*2][N] (feature f of coordinate n at f*N + n), the layout
 * ptycho_cmlp_backward_planar writes.  item_planar holds 2*l*N + n for each
 * item n*n_levels + l of the CSR (same order).  One entry's contributors are
 * spatially adjacent coordinates, so in this layout their gradients are read
 * with coalesced loads.  Results are bitwise those of ptycho_hashgrid_backward.
 * 2*n_levels*N must fit in int32. */
int ptycho_hashgrid_backward_planar(const int32_t* start, const int32_t* item_planar,
                                    const float* weight, const float* dfeatures_planar, int N,
                                    int n_levels, int log2_hashmap_size, int base_resolution,
                                    float per_level_scale, float* dtable, int accumulate,
                                    ptycho_stream_t stream);

/* ---------------------------------------------------------------------- *
 * Complex-exponential MLP on the tensor cores (tcgen05, BF16 operands, FP32
 * accumulation).  Replaces ComplexMLP.net (models/complex_inr.py:6-82,
 * :308-314) for 32 input features, hidden_features 64, hidden_layers 2.
 * ptycho_cmlp_pack converts torch-layout parameters (W1 [32][32] f32,
 * b1 [32] f32, omega1 [1] f32, W2/W3 [32][32] complex64, b2/b3 [32]
 * complex64, omega2/3 [1] f32, Wo [1][32] complex64, bo [1] complex64)
 * into an operand blob of ptycho_cmlp_packed_bytes() bytes.
 * forward: x [N][32] f32 -> y [N] complex64.
 * backward: recomputes the forward and returns, for upstream gy [N]
 * complex64, gx [N][32] (may be NULL), y (may be NULL) and the parameter
 * gradients in `grad` (ptycho_cmlp_grad_floats() floats, torch complex
 * convention): W1 @0 [32][32], b1 @1024, omega1 @1056, W2 @1058 [32][32]
 * complex, b2 @3106 complex, omega2 @3170, W3 @3172, b3 @5220, omega3 @5284,
 * Wo @5286 [32] complex, bo @5350 complex.  Deterministic (per-CTA partial
 * accumulators summed in a fixed order).
 * ---------------------------------------------------------------------- */
size_t ptycho_cmlp_packed_bytes(void);
int ptycho_cmlp_grad_floats(void);
int ptycho_cmlp_pack(const float* W1, const float* b1, const float* omega1, const float* W2,
                     const float* b2, const float* omega2, const float* W3, const float* b3,
                     const float* omega3, const float* Wo, const float* bo, void* packed,
                     ptycho_stream_t stream);
int ptycho_cmlp_forward(const void* packed, const float* x, int N, float* y, int32_t* status_out,
                        ptycho_stream_t stream);
size_t ptycho_cmlp_backward_workspace_size(int N);
int ptycho_cmlp_backward(const void* packed, const float* x, const float* gy, int N, float* gx,
                         float* grad, float* y, void* workspace, size_t workspace_bytes,
                         int32_t* status_out, ptycho_stream_t stream);

/* ptycho_cmlp_forward with x feature-major, x_planar [32][N] (feature f of
 * coordinate n at x_planar[f*N + n]), the layout ptycho_hashgrid_forward_planar
 * writes. */
int ptycho_cmlp_forward_planar(const void* packed, const float* x_planar, int N, float* y,
                               int32_t* status_out, ptycho_stream_t stream);

/* ptycho_cmlp_backward with x and gx feature-major ([32][N], feature f of
 * coordinate n at f*N + n): x as ptycho_hashgrid_forward_planar writes it, gx as
 * ptycho_hashgrid_backward_planar reads it. */
int ptycho_cmlp_backward_planar(const void* packed, const float* x, const float* gy, int N, float* gx,
                                float* grad, float* y, void* workspace, size_t workspace_bytes,
                                int32_t* status_out, ptycho_stream_t stream);

/* ---------------------------------------------------------------------- *
 * Fused Adam step over up to 48 float32 tensors (torch.optim.Adam,
 * Recovery.py:238-241,321; complex parameters as their real view).  The
 * pointer arrays and numels are host arrays; the tensors are device memory.
 * ---------------------------------------------------------------------- */
int ptycho_adam_step(float* const* params, const float* const* grads, float* const* exp_avg,
                     float* const* exp_avg_sq, const long long* numels, int n_tensors, int step,
                     float lr, float beta1, float beta2, float eps, ptycho_stream_t stream);

/* The same step with the step counter (device int32, incremented by the
 * call before use) and the learning rate (device float32) in device memory,
 * so the call can be captured once in a CUDA graph and replayed every step
 * (the torch.optim.Adam(capturable=True) arrangement). */
int ptycho_adam_step_dev(float* const* params, const float* const* grads, float* const* exp_avg,
                         float* const* exp_avg_sq, const long long* numels, int n_tensors,
                         int32_t* step, const float* lr, float beta1, float beta2, float eps,
                         ptycho_stream_t stream);

/* ---------------------------------------------------------------------- *
 * Chain rule through the fused loss: a_out = g * a (na floats) and
 * b_out = g * b (nb floats) in one launch, g = *scale a device double (the
 * upstream gradient autograd hands the fused loss's FP64 output).  Used for dO
 * and dP (complex64 as their float views).  No counterpart in the reference,
 * where autograd scales each gradient inside its own backward graph.
 * ---------------------------------------------------------------------- */
int ptycho_scale_pair(const float* a, float* a_out, long long na, const float* b, float* b_out,
                      long long nb, const double* scale, ptycho_stream_t stream);

/* ---------------------------------------------------------------------- *
 * Residual composition of the INR output, apply_residual of
 * models/complex_inr.py:132-135: out = k * m + init, k a real float32 scalar
 * in device memory, m / init / out complex64 [n].  The backward gives
 * gm = k * g (skipped when gm is null) and *gk = sum Re(conj(g) m), summed in
 * FP64 in a fixed order within one launch.  The workspace
 * (ptycho_residual_workspace_size() bytes, 256-byte aligned) must be zeroed
 * once before its first use; every call leaves it zeroed again.  Calls that
 * share a workspace must not overlap on the GPU.
 * ---------------------------------------------------------------------- */
size_t ptycho_residual_workspace_size(void);

int ptycho_residual(const float* k, const float* m, const float* init, long long n, float* out,
                    ptycho_stream_t stream);

int ptycho_residual_backward(const float* k, const float* m, const float* g, long long n, float* gm,
                             float* gk, void* workspace, size_t workspace_bytes, ptycho_stream_t stream);

/* ---------------------------------------------------------------------- *
 * Fourier upsampling of the INR object.  Replaces fourier_upsample of
 * models/complex_inr.py:252-271 (called at :287):
 *   y = ifft2(ifftshift(pad(fftshift(fft2(x))))) * s^2,
 * x [h][w] complex64 -> y [h*s][w*s] complex64, the pad centred at
 * ((h*s - h)/2, (w*s - w)/2).  The adjoint maps an upstream gradient gy
 * [h*s][w*s] to gx [h][w] (torch's complex convention; the operator's
 * conjugate transpose).  h, w, h*s and w*s must be powers of two in
 * [64, 4096] with s in {1, 2, 4}; otherwise PTYCHO_ERR_UNSUPPORTED_SIZE.
 * workspace: device scratch of ptycho_fourier_upsample_workspace_size()
 * bytes (the intermediate after the row pass), 8-byte aligned.
 * ---------------------------------------------------------------------- */
size_t ptycho_fourier_upsample_workspace_size(int h, int w, int s);

int ptycho_fourier_upsample(const float* x, int h, int w, int s, float* y, void* workspace,
                            size_t workspace_bytes, ptycho_stream_t stream);

int ptycho_fourier_upsample_adjoint(const float* gy, int h, int w, int s, float* gx,
                                    void* workspace, size_t workspace_bytes,
                                    ptycho_stream_t stream);

/* ---------------------------------------------------------------------- *
 * Probe preparation.  Replaces the per-minibatch probe centring and
 * normalisation of Recovery.py:262-285 (utils center_probe's centre-of-mass
 * roll, then scaling to sum |P|^2 = M*N), without host synchronisation:
 *   cp = trunc([M, N]/2 - [M, N] * mean(cumsum(marginal |P|^2)) / tot + 1)
 *   P_out = sqrt(M N / e) * roll(P, -cp),  e = sum |P|^2   (no change if e == 0)
 * P, P_out [M][N] complex64 (distinct buffers), M, N <= 1024.  state [4]
 * doubles receives {cp_y, cp_x, scale, e} for the backward.  Sums are FP64
 * in a fixed order.  The backward maps the gradient of P_out to that of P
 * (torch's complex convention), including the term through e.
 * ---------------------------------------------------------------------- */
int ptycho_probe_center_normalize(const float* P, int M, int N, float* P_out, double* state,
                                  ptycho_stream_t stream);

int ptycho_probe_center_normalize_backward(const float* P_out, const double* state,
                                           const float* grad_out, int M, int N, float* grad_in,
                                           ptycho_stream_t stream);

/* ---------------------------------------------------------------------- *
 * Haar-wavelet sparsity.  Replaces haar_wavelet_sparsity_loss
 * (utils/loss.py:60-83; used at Recovery.py:309-313): the L1 norm of the
 * three detail subbands of the 2x2 Haar transform of img [H][W] complex64
 * (real and imaginary parts separately), as one FP64 value *loss_out
 * (device), summed in a fixed order.  H and W must be even.  workspace:
 * ptycho_haar_sparsity_workspace_size() bytes.  The backward writes
 * grad_img = (*grad_loss) * d loss / d img (torch's complex convention,
 * sign(0) = 0), grad_loss being a device double.
 * ---------------------------------------------------------------------- */
size_t ptycho_haar_sparsity_workspace_size(int H, int W);

int ptycho_haar_sparsity(const float* img, int H, int W, double* loss_out, void* workspace,
                         size_t workspace_bytes, ptycho_stream_t stream);

int ptycho_haar_sparsity_backward(const float* img, int H, int W, const double* grad_loss,
                                  float* grad_img, ptycho_stream_t stream);

/* ---------------------------------------------------------------------- *
 * Object error against ground truth after global-phase alignment, in FP64:
 * over the box [y0, y1) x [x0, x1) of recon and truth ([H][W] complex64),
 * c = sum conj(recon) truth, and with the phase a = arg(c) (the minimiser of
 * ||recon e^{ia} - truth||: resolve_global_phase, scripts/compare_object_ssim.py:92-98),
 *   out[0] = sqrt((sum|recon|^2 + sum|truth|^2 - 2|c|) / sum|truth|^2),
 *   out[1..2] = cos a, sin a,  out[3] = |c|, out[4..5] = the two energies,
 *   out[6] = sqrt(1 - |c|^2 / (sum|recon|^2 sum|truth|^2)), the error after the
 *            least-squares complex factor (phase and scale ambiguity removed).
 * out: 7 device doubles.  Fixed-order sums.  workspace:
 * ptycho_object_error_workspace_size() bytes.
 * ---------------------------------------------------------------------- */
size_t ptycho_object_error_workspace_size(void);

int ptycho_object_error(const float* recon, const float* truth, int H, int W, int y0, int y1, int x0,
                        int x1, double* out, void* workspace, size_t workspace_bytes,
                        ptycho_stream_t stream);

/* ---------------------------------------------------------------------- *
 * 2-D complex Gaussian splatting (the Gaussian-field representation's
 * rasteriser).  Replaces the gscp extension: GaussianRasterize2D /
 * GaussianRasterize2DCholesky (gscp/cuda/_wrapper.py:18-163), i.e.
 * rasterize_forward[_cholesky] / rasterize_backward[_cholesky]
 * (gscp/csrc/rasterize_gaussians.cu, gscp_rasterizer/forward.cu, backward.cu).
 *
 * kind PTYCHO_GS_RS:       p1 = log scales [N][2], p2 = rotation [N] (radians)
 * kind PTYCHO_GS_CHOLESKY: p1 = log diag(L) [N][2], p2 = L21 [N]
 * xy [N][2] pixel positions (x, y), weight [N][2] (re, im); out [2][H][W].
 * Per pixel: sum over the Gaussians whose 16x16-tile rectangle (3-sigma radius,
 * clamped scales in [min_scale, max_patch_radius]) covers the pixel's tile,
 * in ascending index, of weight * exp(power), terms with power > 0 or
 * exp(power) < 1e-7 skipped -- the reference's semantics.  radii_out (int32
 * [N], optional) receives the radii (0 = culled).  No host synchronisation;
 * the workspace (ptycho_gs_workspace_size bytes, 256-byte aligned) carries the
 * per-Gaussian geometry and the per-tile bitmasks from the forward to the
 * backward, which must see the same inputs.  The backward writes every
 * gradient (zeros for culled Gaussians) with fixed-order sums: deterministic.
 * ---------------------------------------------------------------------- */
enum { PTYCHO_GS_RS = 0, PTYCHO_GS_CHOLESKY = 1 };

size_t ptycho_gs_workspace_size(int N, int H, int W);

int ptycho_gs_forward(int kind, const float* xy, const float* p1, const float* p2, const float* weight,
                      int N, int H, int W, int max_patch_radius, float min_scale, float* out,
                      int* radii_out, void* workspace, size_t workspace_bytes, ptycho_stream_t stream);

int ptycho_gs_backward(int kind, const float* xy, const float* p1, const float* p2, const float* weight,
                       int N, int H, int W, int max_patch_radius, float min_scale, const float* grad_out,
                       const void* workspace, size_t workspace_bytes, float* dxy, float* dp1, float* dp2,
                       float* dweight, ptycho_stream_t stream);

/* ---------------------------------------------------------------------- *
 * Hash-grid backward for coordinates on a tensor-product grid (an INR's pixel
 * centres, models/complex_inr.py:179-205): coordinate n = i * Bj + j is
 * (ax0[j], ax1[i]) with both axes non-decreasing.  Same result as
 * ptycho_hashgrid_backward (the table gradient, deterministic), without the
 * per-contribution CSR: every level's vertex sums the rectangle of
 * coordinates whose cells touch it, then every entry sums its vertices.
 * extents: HOST [n_levels][4] int32 per level: vertex extents E0, E1 and the
 *   most axis values in one cell along each axis (cw0, cw1).  Coarse levels
 *   (cw0 * cw1 >= 16) are summed separably: a row pass forms per row and
 *   cell S0 = sum (1 - fx) g and S1 = sum fx g, a column pass sums
 *   wy (S1[cx - 1] + S0[cx]) over the rows of each vertex; finer levels per
 *   vertex from shared-memory tiles.
 * grid_int (device int32): ix0 [L][Bj], iy1 [L][A] (cell corners of the axis
 *   values), lo0 [sum (E0+1)], lo1 [sum (E1+1)] (first axis index whose corner
 *   is >= c), vstart [entries+1], vorder [vertices] (vertices sorted by entry);
 * grid_frac (device float32): fx0 [L][Bj], fy1 [L][A] (cell fractions of
 *   x * scale + 0.5 formed with one rounding).
 * scratch: ptycho_hashgrid_grid_scratch_size(extents, n_levels, A, Bj) bytes.
 * dfeatures [N][2L] or, with planar, feature-major [2L][N].
 * ---------------------------------------------------------------------- */
size_t ptycho_hashgrid_grid_scratch_size(const int32_t* extents, int n_levels, int A, int Bj);

int ptycho_hashgrid_backward_grid(const int32_t* grid_int, const float* grid_frac, const int32_t* extents, int A,
                                  int Bj, const float* dfeatures, int planar, int n_levels, int log2_hashmap_size,
                                  int base_resolution, float per_level_scale, float* dtable, int accumulate,
                                  void* scratch, size_t scratch_bytes, ptycho_stream_t stream);

/* ---------------------------------------------------------------------- *
 * ptycho_fwd_adj without a workspace, for callers that cannot allocate
 * device memory (an FFI host with no CUDA allocator of its own, a step that
 * must not trigger an allocation's device synchronisation).  No counterpart
 * in the reference.  Same arguments and results as ptycho_fwd_adj minus the
 * workspace: the scratch is a 48 MiB static device array inside this
 * library, held by every GPU that loads it until the process exits.  A call
 * needing more than 48 MiB of scratch (ptycho_fwd_adj_workspace_size) returns
 * PTYCHO_ERR_WORKSPACE without touching the device (M = 128 fits up to about
 * 360 patterns per call).  Arguments ptycho_fwd_adj refuses get its status
 * first, before any lookup.  Every call looks up the array's address in the
 * current context (an address cached from another context could be stale);
 * the first call in a context may load the module, so make it before any
 * stream capture.  All calls share the array: calls that overlap on the GPU
 * race, so order them on one stream.
 * ---------------------------------------------------------------------- */
int ptycho_fwd_adj_noalloc(const float* O, int H, int W, const float* P, int M, int N,
                           const int32_t* tl, const float* Imeas, int F, const int32_t* batch,
                           int B, int loss_type, double* loss_per_pattern, double* loss_total,
                           float* dO, float* dP, unsigned flags, int32_t* status_out,
                           ptycho_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* PTYCHO_B200_H */
