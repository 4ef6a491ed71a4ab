// TEST ONLY -- a C entry point onto the reference's own Gaussian rasteriser
// (gscp/csrc/gscp_rasterizer: forward.cu, backward.cu, rasterizer_impl.cu),
// compiled from those sources where they lie by oracle/build_ref.py into
// oracle/_ref/libgscp_ref.so.  The parity tests call it as the checker for
// ptycho_gs_forward / ptycho_gs_backward.  Nothing in the product links it.
//
// The reference grows its geometry / binning / image buffers through
// std::function allocators (torch tensors in gscp/csrc/rasterize_gaussians.cu);
// here they are cudaMalloc'ed and kept in a handle between the forward and the
// backward.  Arguments are device pointers, float32, in the reference's layout.
#include <cuda_runtime.h>

#include <cstdio>
#include <functional>

#include "rasterizer.h"

namespace {

struct Buf {
  char* p = nullptr;
  size_t n = 0;
  std::function<char*(size_t)> fn() {
    return [this](size_t sz) -> char* {
      if (sz > n) {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        if (cudaMalloc(&p, sz ? sz : 1) != cudaSuccess) return nullptr;
        n = sz;
      }
      return p;
    };
  }
  ~Buf() {
    if (p) cudaFree(p);
  }
};

struct Handle {
  Buf geom, binning, img;
  int rendered = 0;
};

}  // namespace

extern "C" {

void* gscp_ref_create(void) { return new Handle(); }

void gscp_ref_destroy(void* h) { delete static_cast<Handle*>(h); }

// kind 0: p1 = log scales [N][2], p2 = rotation [N]; kind 1: p1 = log diag(L), p2 = L21.
int gscp_ref_forward(void* h, int kind, int N, int H, int W, const float* xy, const float* p1, const float* p2,
                     const float* weight, int max_patch_radius, float min_scale, float* out, int* radii) {
  Handle* hd = static_cast<Handle*>(h);
  cudaMemset(out, 0, sizeof(float) * 2 * H * W);
  if (N == 0) return 0;
  if (kind == 0)
    hd->rendered = GscpRasterizer::Rasterizer::forward(hd->geom.fn(), hd->binning.fn(), hd->img.fn(), N, W, H, xy,
                                                       p1, p2, weight, max_patch_radius, min_scale, out, radii,
                                                       false);
  else
    hd->rendered = GscpRasterizer::Rasterizer::forward_cholesky(hd->geom.fn(), hd->binning.fn(), hd->img.fn(), N, W,
                                                                H, xy, p1, p2, weight, max_patch_radius, min_scale,
                                                                out, radii, false);
  return cudaGetLastError() == cudaSuccess ? hd->rendered : -1;  // stream-ordered like the reference
}

// Gradients are accumulated by the reference with atomicAdd: the outputs and
// the two scratch arrays (dmean [N][2], dconic [N][3]) must be zeroed first.
int gscp_ref_backward(void* h, int kind, int N, int H, int W, const float* xy, const float* p1, const float* p2,
                      const float* weight, int max_patch_radius, float min_scale, const int* radii,
                      const float* grad_out, float* dmean, float* dconic, float* dweight, float* dxy, float* dp1,
                      float* dp2) {
  Handle* hd = static_cast<Handle*>(h);
  if (N == 0 || hd->rendered == 0) return 0;
  if (kind == 0)
    GscpRasterizer::Rasterizer::backward(N, hd->rendered, W, H, xy, p1, p2, weight, max_patch_radius, min_scale,
                                         radii, hd->geom.p, hd->binning.p, hd->img.p, grad_out, dmean, dconic,
                                         dweight, dxy, dp1, dp2, false);
  else
    GscpRasterizer::Rasterizer::backward_cholesky(N, hd->rendered, W, H, xy, p1, p2, weight, max_patch_radius,
                                                  min_scale, radii, hd->geom.p, hd->binning.p, hd->img.p, grad_out,
                                                  dmean, dconic, dweight, dxy, dp1, dp2, false);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // extern "C"
