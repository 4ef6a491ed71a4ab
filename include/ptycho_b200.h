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
  PTYCHO_ERR_UNSUPPORTED_SIZE = 2, /* probe size not in {64,128,256}, M != N */
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
 * Supported: M == N in {64, 128}.  Needs no scratch memory.
 * ---------------------------------------------------------------------- */
int ptycho_forward_intensity(const float* O, int H, int W, const float* P, int M, int N,
                             const int32_t* tl, int F, const int32_t* batch, int B,
                             float* I_out, int32_t* status_out, ptycho_stream_t stream);

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
 * ---------------------------------------------------------------------- */
size_t ptycho_fwd_adj_workspace_size(int H, int W, int M, int N, int B);

int ptycho_fwd_adj(const float* O, int H, int W, const float* P, int M, int N,
                   const int32_t* tl, const float* Imeas, int F, const int32_t* batch, int B,
                   int loss_type, double* loss_per_pattern, double* loss_total, float* dO,
                   float* dP, unsigned flags, void* workspace, size_t workspace_bytes,
                   int32_t* status_out, ptycho_stream_t stream);

/* ---------------------------------------------------------------------- *
 * ptycho_fwd_adj without a workspace, for callers that cannot allocate
 * device memory (an FFI host with no CUDA allocator of its own, a step that
 * must not trigger an allocation's device synchronisation).  No counterpart
 * in the reference.  Same arguments and results as ptycho_fwd_adj minus the
 * workspace: the scratch is a 48 MiB static device array inside this
 * library, held by every GPU that loads it until the process exits.  A call
 * needing more than 48 MiB of scratch (ptycho_fwd_adj_workspace_size) returns
 * PTYCHO_ERR_WORKSPACE without touching the device (M = 128 fits up to about
 * 360 patterns per call).  The first call on a device looks up the array's
 * address; make it before any stream capture.  All calls share the array:
 * calls that overlap on the GPU race, so order them on one stream.
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
