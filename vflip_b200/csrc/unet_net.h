// Host side of the learned preconditioner's 3D U-Net (internal C++ interface
// shared by the library's translation units; the C ABI is in vflip.h).
//
// Architecture (4 levels, 16/32/64/128 channels, 3x3x3 convolutions, ReLU,
// 2x2x2 average pooling, nearest upsampling, skip connections by
// concatenation):
//   in(16: rhs, fluid fraction, 14 zero) -E0A-> 16 -E0B-> 16 ------------------------------+
//     pool -E1A-> 32 -E1B-> 32 ------------------------------------------------+            |
//       pool -E2A-> 64 -E2B-> 64 ---------------------------------+            |            |
//         pool -B1-> 128 -B2-> 128 -up-> [128 | 64] -D2A-> 64 -D2B-> 64 -up-> [64 | 32] -D1A-> 32 -D1B-> 32
//           -up-> [32 | 16] -D0A-> 16 -D0B-> 16 -OUT-> 2 (warm-start pressure, coarse correction)
// Parameters are FP32 masters (W[cout][cin][27], b[cout] per layer, in layer
// order); the convolutions run on BF16 copies packed for the tensor-core
// kernels.  Grid dimensions must be multiples of 8 (three poolings).
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace vflip {
namespace unet {

enum Layer { E0A, E0B, E1A, E1B, E2A, E2B, B1, B2, D2A, D2B, D1A, D1B, D0A, D0B, OUT, kNumLayers };
struct LayerSpec {
  int cin, cout, relu;
};
extern const LayerSpec kSpec[kNumLayers];
constexpr int kOutValid = 2;  // OUT computes 16 channels, only the first 2 have weights

struct View {
  __nv_bfloat16* p;
  int ctot, coff, c;
};

class Net {
 public:
  Net(int device, cudaStream_t stream, unsigned long long seed);
  ~Net();
  int init_status() const { return init_rc; }

  int forward(int X, int Y, int Z, const float* in2, float* out2);
  // The same forward pass replayed as a CUDA graph, captured once per
  // (grid, buffers) and launched on `stream`: the inference path, whose
  // ~30 launches would otherwise each pay a host-side launch and
  // tensor-map encode.  Bitwise the eager pass.
  int forward_replay(int X, int Y, int Z, const float* in2, float* out2);
  int backward(const float* target2, const float* weight, float cw0, float cw1, double* loss);
  int adam(float lr, float b1 = 0.9f, float b2 = 0.999f, float eps = 1e-8f);
  int repack();
  int get_params(float* host) const;
  int set_params(const float* host);
  int copy_grads(float* dst) const;
  int sync_error();  // reads the kernels' error flag (synchronises the stream)

  // single operations (also used by the tests)
  int conv(const View& in, int X, int Y, int Z, const __nv_bfloat16* wpacked, const float* bias, int cin, int cout,
           int relu, const View* mask, const View* out, float* outf, int ofstride, int ofvalid);
  int wgrad(const View& x, const View& dy, int X, int Y, int Z, int cin, int cout, float* dw_master);
  int channel_sum(const View& g, size_t nvox, float* out);
  int pack(const float* w, __nv_bfloat16* out, int cin, int cout, int flip);

  int fail(int code, const char* fmt, ...);
  void* scratch(size_t bytes, int slot);  // slot-keyed device workspace (grows)

  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  int num_sms = 148;
  int nparams = 0;
  size_t woff[kNumLayers] = {}, boff[kNumLayers] = {};
  float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
  __nv_bfloat16 *wf[kNumLayers] = {}, *wd[kNumLayers] = {};
  int adam_t = 0;
  float out_scale[2] = {1.0f, 1.0f};  // multiplies the two outputs when the solver uses them
  long long launches = 0;
  int* d_error = nullptr;

 private:
  int init_rc = 0;
  int ensure_acts(int X, int Y, int Z);
  struct Acts;
  Acts* acts = nullptr;
  std::vector<std::pair<void*, size_t>> scratch_;
  void* act_mem = nullptr;
  size_t act_bytes = 0;
  cudaStream_t cap_stream = nullptr;  // capture stream of forward_replay
  cudaGraph_t fwd_graph = nullptr;
  cudaGraphExec_t fwd_exec = nullptr;
  std::vector<uintptr_t> fwd_key;
  long long fwd_launches = 0;
};

}  // namespace unet
}  // namespace vflip

// the C ABI handle (include/vflip.h)
struct vflip_unet {
  vflip::unet::Net* net;
};
