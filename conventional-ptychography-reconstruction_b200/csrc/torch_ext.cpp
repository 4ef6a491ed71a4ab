// torch_ext.cpp -- the fused loss as a C++ torch autograd function over the C ABI.
//
// fused_loss (Recovery.py:288-307, backward at :316) needs an autograd node
// whose backward scales the gradients the forward already computed.  Written
// in Python, every step pays the Python Function machinery twice (forward and,
// from the autograd engine's thread, backward).  Here the node is C++: the
// forward calls ptycho_fwd_adj, the backward ptycho_scale_pair, both through
// addresses handed over by `bind` (taken from the ctypes handle of
// libptycho_b200.so, so there is one copy of the library in the process).
// No computation happens here; a non-zero library status raises RuntimeError,
// bad arguments raise ValueError / TypeError as the Python path does.
#include <ATen/cuda/CUDAContext.h>
#include <c10/cuda/CUDAGuard.h>
#include <torch/extension.h>

#include <cstdint>
#include <mutex>
#include <optional>
#include <unordered_map>

namespace {

using torch::Tensor;
using torch::autograd::AutogradContext;
using torch::autograd::tensor_list;

typedef int (*fwd_adj_fn)(const float*, int, int, const float*, int, int, const int32_t*, const float*, int,
                          const int32_t*, int, int, double*, double*, float*, float*, unsigned, void*, size_t,
                          int32_t*, void*);
typedef int (*scale_pair_fn)(const float*, float*, long long, const float*, float*, long long, const double*,
                             void*);
typedef size_t (*ws_size_fn)(int, int, int, int, int);
typedef const char* (*status_string_fn)(int);

fwd_adj_fn g_fwd_adj = nullptr;
scale_pair_fn g_scale_pair = nullptr;
ws_size_fn g_ws_size = nullptr;
status_string_fn g_status_string = nullptr;

constexpr int64_t kMaxProbeDim = 4096;

void check(int rc, const char* where) {
  TORCH_CHECK(rc == 0, where, ": ", g_status_string ? g_status_string(rc) : "error", " (status ", rc, ")");
}

template <typename T>
T* fptr(const Tensor& t) {
  return t.defined() ? reinterpret_cast<T*>(t.data_ptr()) : nullptr;
}

// One growing workspace per (device, stream): calls on one stream are ordered,
// calls on different streams must not share scratch.  The Python entry points
// use the same cache, so a process holds one workspace per stream.
std::mutex g_ws_mu;
std::unordered_map<uint64_t, Tensor> g_ws;

// At most kMaxWorkspaces entries: a caller that keeps creating streams would
// otherwise keep every old stream's workspace alive.  Dropping an entry is
// safe: each workspace was allocated on its own stream, and the caching
// allocator reuses freed memory in that stream's order.
constexpr size_t kMaxWorkspaces = 16;

Tensor workspace_on(const Tensor& like, cudaStream_t s, size_t bytes) {
  const uint64_t key = (uint64_t(like.device().index()) << 56) ^ reinterpret_cast<uintptr_t>(s);
  std::lock_guard<std::mutex> lock(g_ws_mu);
  if (g_ws.size() >= kMaxWorkspaces && g_ws.find(key) == g_ws.end()) g_ws.clear();
  Tensor& w = g_ws[key];
  if (!w.defined() || size_t(w.numel()) < bytes)
    w = torch::empty({int64_t(bytes < 256 ? 256 : bytes)}, like.options().dtype(torch::kUInt8));
  return w;
}

cudaStream_t current_stream(const Tensor& t) {
  return at::cuda::getCurrentCUDAStream(t.device().index()).stream();
}

// Nothing throws inside the node's forward: the wrapper below checks and
// converts every argument before apply(), and a library error is handed out
// through `rc` and raised after apply() has returned.
class FusedLoss : public torch::autograd::Function<FusedLoss> {
 public:
  // O [H, W] c64, P [M, N] c64 on one CUDA device; tl [F, 2] int32, Imeas
  // [F, M, N] float32, batch [B] int32 frame ids (none: all F frames) and the
  // status word [1] int32, all contiguous on that device.  The batch is an
  // optional (not an undefined tensor): autograd records a device for every
  // tensor argument.
  static Tensor forward(AutogradContext* ctx, Tensor O, Tensor P, const Tensor& tl, const Tensor& Imeas,
                        int64_t loss_code, const std::optional<Tensor>& batch, const Tensor& status, bool need_grad,
                        int* rc) {
    O = O.contiguous();
    P = P.contiguous();
    const int64_t H = O.size(0), W = O.size(1), M = P.size(0), N = P.size(1);
    const int64_t F = tl.size(0);
    const bool has_batch = batch.has_value() && batch->defined();
    const int64_t B = has_batch ? batch->numel() : F;
    cudaStream_t s = current_stream(O);
    Tensor loss = torch::empty({}, O.options().dtype(torch::kFloat64));
    Tensor dO, dP;
    if (need_grad) {
      dO = torch::empty({H, W}, O.options());
      dP = torch::empty({M, N}, P.options());
    }
    Tensor ws = workspace_on(O, s, g_ws_size(int(H), int(W), int(M), int(N), int(B)));
    *rc = g_fwd_adj(fptr<const float>(O), int(H), int(W), fptr<const float>(P), int(M), int(N),
                    fptr<const int32_t>(tl), fptr<const float>(Imeas), int(F),
                    has_batch ? fptr<const int32_t>(*batch) : nullptr, int(B), int(loss_code), nullptr,
                    fptr<double>(loss), fptr<float>(dO), fptr<float>(dP), 0u, ws.data_ptr(), size_t(ws.numel()),
                    fptr<int32_t>(status), s);
    ctx->save_for_backward({dO, dP});
    return loss;
  }

  static tensor_list backward(AutogradContext* ctx, tensor_list grads) {
    auto saved = ctx->get_saved_variables();
    const Tensor& dO = saved[0];
    const Tensor& dP = saved[1];
    const bool nO = ctx->needs_input_grad(0) && dO.defined() && grads[0].defined();
    const bool nP = ctx->needs_input_grad(1) && dP.defined() && grads[0].defined();
    Tensor gO, gP;
    if (nO || nP) {
      Tensor g = grads[0].to(torch::kFloat64).contiguous();
      gO = nO ? torch::empty_like(dO) : Tensor();
      gP = nP ? torch::empty_like(dP) : Tensor();
      // one launch scales both (out of place: the saved gradients stay valid for a second backward)
      check(g_scale_pair(nO ? fptr<const float>(dO) : nullptr, fptr<float>(gO), nO ? 2 * dO.numel() : 0,
                         nP ? fptr<const float>(dP) : nullptr, fptr<float>(gP), nP ? 2 * dP.numel() : 0,
                         fptr<const double>(g), current_stream(g)),
            "ptycho_scale_pair");
    }
    return {gO, gP, Tensor(), Tensor(), Tensor(), Tensor(), Tensor(), Tensor(), Tensor()};
  }
};

void bind(int64_t fwd_adj, int64_t scale_pair, int64_t ws_size, int64_t status_string) {
  g_fwd_adj = reinterpret_cast<fwd_adj_fn>(fwd_adj);
  g_scale_pair = reinterpret_cast<scale_pair_fn>(scale_pair);
  g_ws_size = reinterpret_cast<ws_size_fn>(ws_size);
  g_status_string = reinterpret_cast<status_string_fn>(status_string);
}

// fused_loss(O, P, tl, Imeas, loss_code, batch|None, status): the caller has
// checked the loss name and the complex64 dtypes
Tensor fused_loss(const Tensor& O, const Tensor& P, const Tensor& tl_in, const Tensor& Imeas_in,
                  int64_t loss_code, const std::optional<Tensor>& batch_in, const Tensor& status) {
  TORCH_CHECK(g_fwd_adj && g_scale_pair && g_ws_size, "bind() was not called");
  TORCH_CHECK_VALUE(O.is_cuda() && P.is_cuda(), "object and probe must be CUDA tensors (there is no CPU path)");
  TORCH_CHECK_VALUE(P.device() == O.device(), "object and probe must be on one device");
  TORCH_CHECK_TYPE(O.scalar_type() == torch::kComplexFloat && P.scalar_type() == torch::kComplexFloat,
                   "object and probe must be complex64");
  TORCH_CHECK_VALUE(O.dim() == 2, "object must be [H, W]");
  TORCH_CHECK_VALUE(P.dim() == 2 && P.size(0) >= 1 && P.size(0) <= kMaxProbeDim && P.size(1) >= 1 &&
                        P.size(1) <= kMaxProbeDim,
                    "probe must be [M, N] with 1 <= M, N <= ", kMaxProbeDim, ", got ", P.sizes());
  TORCH_CHECK_VALUE(status.is_cuda() && status.device() == O.device() && status.scalar_type() == torch::kInt32,
                    "status must be the device's int32 status word");
  const auto dev = O.device();
  c10::cuda::CUDAGuard guard(dev);
  // windows, measurements and frame ids carry no gradient (the node returns none for them)
  const Tensor tl = tl_in.detach().to(dev, torch::kInt32).contiguous();
  const Tensor Imeas = Imeas_in.detach().to(dev, torch::kFloat32).contiguous();
  std::optional<Tensor> batch;
  if (batch_in.has_value() && batch_in->defined()) batch = batch_in->detach().to(dev, torch::kInt32).contiguous();
  const int64_t F = tl.dim() == 2 ? tl.size(0) : -1;
  TORCH_CHECK_VALUE(tl.dim() == 2 && tl.size(1) == 2, "windows must be [F, 2] (tlY, tlX)");
  TORCH_CHECK_VALUE(Imeas.dim() == 3 && Imeas.size(0) == F && Imeas.size(1) == P.size(0) &&
                        Imeas.size(2) == P.size(1),
                    "measurements must be [F, M, N] = (", F, ", ", P.size(0), ", ", P.size(1), "), got ",
                    Imeas.sizes());
  const bool need = torch::GradMode::is_enabled() && (O.requires_grad() || P.requires_grad());
  int rc = 0;
  Tensor loss = FusedLoss::apply(O, P, tl, Imeas, loss_code, batch, status, need, &rc);
  check(rc, "ptycho_fwd_adj");
  return loss;
}

// the cached workspace of the current stream of `like`'s device, at least `bytes` long
Tensor workspace(const Tensor& like, int64_t bytes) {
  TORCH_CHECK_VALUE(like.is_cuda() && bytes >= 0, "workspace needs a CUDA tensor and a size");
  return workspace_on(like, current_stream(like), size_t(bytes));
}

}  // namespace

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
  m.def("bind", &bind, "bind(fwd_adj, scale_pair, workspace_size, status_string) function addresses");
  m.def("fused_loss", &fused_loss, "fused forward + loss + adjoint as one autograd node");
  m.def("workspace", &workspace, "the per-stream ptycho_fwd_adj workspace");
}
