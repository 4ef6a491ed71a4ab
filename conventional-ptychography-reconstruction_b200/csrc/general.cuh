// general.cuh -- the any-size probe path (general.cu).
#pragma once
#include "fused.cuh"

namespace pty {

constexpr int kGeneralMaxDim = 4096;  // largest probe side the general path takes

bool general_supported(int M, int N);

// |fftshift(fft2(P * O_window))|^2 for a.B patterns into a.I_out; X: [B][M][N] scratch
int general_forward_intensity(const FusedArgs& a, int M, int N, float2* X, cudaStream_t s);

// per-pattern losses into a.loss_pat; with grad, X ends as E_b = dL/dpsi_b
// (no fftshift sign) and tlb holds the resolved windows ((-1,-1): skipped).
// scr: 3 * B * M * N floats (FD loss)
int general_fwd_adj(const FusedArgs& a, int M, int N, int loss, bool grad, float2* X, float* scr, int2* tlb,
                    cudaStream_t s);

}  // namespace pty
