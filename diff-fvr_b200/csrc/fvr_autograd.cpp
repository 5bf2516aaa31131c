// Native autograd binding of the spectral-NCC value-and-gradient launch.
//
// The reference's loss (src/fvr/torch_engine.py:292-307, forward_spectral_ncc)
// is differentiated by PyTorch's autograd.  Here the forward pass already
// computes the pose gradient (the moments kernel and its dependent epilogue,
// fvr_tc_sncc_value_and_grad in libfvr_b200.so), so the autograd node only has
// to keep dL/dposes and scale it by the upstream gradient.  Written as a C++
// torch::autograd::Function, one forward call costs one pybind call, two
// allocations and the foreign launch, and the backward runs on the autograd
// engine's device thread without taking the Python interpreter lock.
//
// The launch itself is reached through the C ABI only: the Python side hands
// over the address of fvr_tc_sncc_value_and_grad and every argument that is
// fixed for a prepared call (stencil storage, shape, views, target spectra,
// high-pass table, launch variant, workspace); this file holds no kernels.
#include <torch/extension.h>
#include <c10/cuda/CUDAStream.h>

#include <cstdint>
#include <string>
#include <vector>

namespace {

using SnccValueAndGrad = int (*)(int, const void*, const float*, int64_t, int64_t, int64_t, const float*, int64_t,
                                 int, const int*, const void* const*, const float*, const float*, int64_t, double,
                                 int, const float*, int64_t, void*, int64_t, float*, float*, float*, int, void*);
using StatusString = const char* (*)(int);

// One prepared launch: the arguments of fvr_tc_sncc_value_and_grad that do
// not change between calls, and the tensors that own the memory they name.
struct SnccCall {
  SnccValueAndGrad fn = nullptr;
  StatusString status = nullptr;
  int dtype = 0;
  const void* stencil = nullptr;
  const float* scales = nullptr;
  int64_t D = 0, H = 0, W = 0, C = 0, R = 0;
  std::vector<int> views;
  std::vector<const void*> ftargs;
  const float* hp = nullptr;
  const float* lin = nullptr;
  double kappa = 0.0;
  int variant = 0;
  void* ws = nullptr;
  int64_t ws_bytes = 0;
  int device = 0;
  std::vector<at::Tensor> keep;
};

template <typename T>
T as_ptr(int64_t v) {
  return reinterpret_cast<T>(static_cast<intptr_t>(v));
}

class SnccLoss : public torch::autograd::Function<SnccLoss> {
 public:
  // Returns sum_v loss_v as a 0-dim tensor; keeps dL/dposes for backward.
  static at::Tensor forward(torch::autograd::AutogradContext* ctx, const at::Tensor& poses, int64_t handle) {
    const SnccCall& k = *as_ptr<const SnccCall*>(handle);
    at::Tensor p = poses.detach();
    if (!p.is_cuda() || p.get_device() != k.device || p.scalar_type() != at::kFloat)
      p = p.to(at::Device(at::kCUDA, static_cast<c10::DeviceIndex>(k.device)), at::kFloat);
    p = p.contiguous();
    TORCH_CHECK(p.dim() == 2 && p.size(0) == k.C && p.size(1) == 6, "poses must have shape (", k.C, ", 6)");
    const auto opts = at::TensorOptions().dtype(at::kFloat).device(at::kCUDA, k.device);
    const int nv = static_cast<int>(k.views.size());
    at::Tensor grad = at::empty({k.C, 6}, opts);
    at::Tensor loss = at::empty({nv + 1}, opts);
    cudaStream_t s = c10::cuda::getCurrentCUDAStream(static_cast<c10::DeviceIndex>(k.device)).stream();
    const int rc = k.fn(k.dtype, k.stencil, k.scales, k.D, k.H, k.W, p.data_ptr<float>(), k.C, nv, k.views.data(),
                        k.ftargs.data(), k.hp, k.lin, k.R, k.kappa, k.variant, nullptr, 0, k.ws, k.ws_bytes,
                        loss.data_ptr<float>(), nullptr, grad.data_ptr<float>(), 0, s);
    TORCH_CHECK(rc == 0, "fvr_tc_sncc_value_and_grad failed with status ", rc, ": ",
                k.status ? k.status(rc) : "");
    ctx->save_for_backward({grad});
    ctx->saved_data["pdt"] = static_cast<int64_t>(poses.scalar_type());
    return loss.select(0, nv);
  }

  // dL/dposes scaled by the upstream gradient of the (scalar) loss.
  static torch::autograd::variable_list backward(torch::autograd::AutogradContext* ctx,
                                                 torch::autograd::variable_list go) {
    at::Tensor grad = ctx->get_saved_variables()[0];
    at::Tensor r = go[0].defined() ? grad * go[0].to(grad.scalar_type()) : at::zeros_like(grad);
    const auto pdt = static_cast<at::ScalarType>(ctx->saved_data["pdt"].toInt());
    if (r.scalar_type() != pdt) r = r.to(pdt);
    return {r, at::Tensor()};
  }
};

at::Tensor sncc_loss(const at::Tensor& poses, const SnccCall& call) {
  return SnccLoss::apply(poses, reinterpret_cast<int64_t>(&call));
}

}  // namespace

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
  m.doc() = "Native autograd binding of fvr_tc_sncc_value_and_grad (libfvr_b200.so)";
  pybind11::class_<SnccCall>(m, "SnccCall")
      .def(pybind11::init([](int64_t fn, int64_t status, int dtype, int64_t stencil, int64_t scales, int64_t D,
                             int64_t H, int64_t W, int64_t C, std::vector<int> views, std::vector<int64_t> ftargs,
                             int64_t hp, int64_t lin, int64_t R, double kappa, int variant, int64_t ws,
                             int64_t ws_bytes, int device, std::vector<at::Tensor> keep) {
             TORCH_CHECK(fn != 0 && stencil != 0 && lin != 0 && ws != 0, "null pointer in a prepared launch");
             TORCH_CHECK(!views.empty() && views.size() == ftargs.size(), "one target spectrum per view");
             auto* k = new SnccCall();
             k->fn = as_ptr<SnccValueAndGrad>(fn);
             k->status = as_ptr<StatusString>(status);
             k->dtype = dtype;
             k->stencil = as_ptr<const void*>(stencil);
             k->scales = as_ptr<const float*>(scales);
             k->D = D;
             k->H = H;
             k->W = W;
             k->C = C;
             k->R = R;
             k->views = std::move(views);
             for (int64_t f : ftargs) k->ftargs.push_back(as_ptr<const void*>(f));
             k->hp = as_ptr<const float*>(hp);
             k->lin = as_ptr<const float*>(lin);
             k->kappa = kappa;
             k->variant = variant;
             k->ws = as_ptr<void*>(ws);
             k->ws_bytes = ws_bytes;
             k->device = device;
             k->keep = std::move(keep);
             return k;
           }),
           pybind11::arg("fn"), pybind11::arg("status"), pybind11::arg("dtype"), pybind11::arg("stencil"),
           pybind11::arg("scales"), pybind11::arg("D"), pybind11::arg("H"), pybind11::arg("W"), pybind11::arg("C"),
           pybind11::arg("views"), pybind11::arg("ftargs"), pybind11::arg("hp"), pybind11::arg("lin"),
           pybind11::arg("R"), pybind11::arg("kappa"), pybind11::arg("variant"), pybind11::arg("ws"),
           pybind11::arg("ws_bytes"), pybind11::arg("device"), pybind11::arg("keep"));
  m.def("sncc_loss", &sncc_loss, "sum_v spectral-NCC loss of the prepared call; differentiable in poses",
        pybind11::arg("poses"), pybind11::arg("call"));
}
