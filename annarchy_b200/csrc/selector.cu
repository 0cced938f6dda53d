// Learned storage-format selector: a small multilayer perceptron trained and
// evaluated on the GPU with hand-written kernels.
//
// The network maps features of a projection's connectivity matrix (row-length
// statistics, density, block fill, weight bytes) to the predicted log10 time
// of the weighted sum under every candidate schedule (format + parameter);
// the selector picks the schedule with the smallest prediction. Layers:
// in -> H (ReLU) -> H (ReLU) -> out (linear). Training minimises the mean
// squared error over the schedules that were measured for a sample (mask).
//
// Parameter layout (float, one contiguous vector):
//   W1[H][in], b1[H], W2[H][H], b2[H], W3[out][H], b3[out]
//
// No counterpart in the reference, which selects formats with a fixed rule
// (ANNarchy/core/Projection.py:691-789).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/annarchy_b200.h"

namespace {

thread_local std::string g_sel_error;

int sel_fail(int code, const std::string& msg) {
  g_sel_error = msg;
  return code;
}

#define SEL_CUDA(call)                                                                     \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) return sel_fail(ANB_ERR_CUDA, std::string(#call) + ": " +       \
                                                             cudaGetErrorString(e_));      \
  } while (0)

struct Dims {
  int in, hidden, out;
  size_t w1() const { return 0; }
  size_t b1() const { return (size_t)hidden * in; }
  size_t w2() const { return b1() + hidden; }
  size_t b2() const { return w2() + (size_t)hidden * hidden; }
  size_t w3() const { return b2() + hidden; }
  size_t b3() const { return w3() + (size_t)out * hidden; }
  size_t total() const { return b3() + out; }
};

// y[b][o] = act(sum_i x[b][i] * W[o][i] + bias[o]); thread per (b, o).
__global__ void linear_fwd(const float* __restrict__ x, const float* __restrict__ W,
                           const float* __restrict__ bias, float* __restrict__ y, int n, int in,
                           int out, int relu) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n * out) return;
  const int b = k / out, o = k % out;
  float s = bias[o];
  const float* xr = x + (size_t)b * in;
  const float* wr = W + (size_t)o * in;
  for (int i = 0; i < in; ++i) s += xr[i] * wr[i];
  y[k] = relu ? fmaxf(s, 0.f) : s;
}

// d[b][o] = 2 * mask * (y - t) / count; loss partial sums per thread block.
__global__ void mse_grad(const float* __restrict__ y, const float* __restrict__ t,
                         const float* __restrict__ mask, float* __restrict__ d, int n, int out,
                         float inv_count, float* __restrict__ loss) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (k < n * out) {
    const float e = (y[k] - t[k]) * mask[k];
    d[k] = 2.f * e * inv_count;
    l = e * e * inv_count;
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0 && l != 0.f) atomicAdd(loss, l);
}

// dx[b][i] = sum_o d[b][o] * W[o][i], then times relu'(x) if `relu_of_x`.
__global__ void linear_bwd_x(const float* __restrict__ d, const float* __restrict__ W,
                             const float* __restrict__ x, float* __restrict__ dx, int n, int in,
                             int out, int relu_of_x) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n * in) return;
  const int b = k / in, i = k % in;
  float s = 0.f;
  for (int o = 0; o < out; ++o) s += d[(size_t)b * out + o] * W[(size_t)o * in + i];
  if (relu_of_x && x[k] <= 0.f) s = 0.f;
  dx[k] = s;
}

// dW[o][i] = sum_b d[b][o] * x[b][i]; db[o] = sum_b d[b][o]. Thread per (o, i)
// (i == in is the bias).
__global__ void linear_bwd_w(const float* __restrict__ d, const float* __restrict__ x,
                             float* __restrict__ dW, float* __restrict__ db, int n, int in,
                             int out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= out * (in + 1)) return;
  const int o = k / (in + 1), i = k % (in + 1);
  float s = 0.f;
  if (i < in) {
    for (int b = 0; b < n; ++b) s += d[(size_t)b * out + o] * x[(size_t)b * in + i];
    dW[(size_t)o * in + i] = s;
  } else {
    for (int b = 0; b < n; ++b) s += d[(size_t)b * out + o];
    db[o] = s;
  }
}

__global__ void adam_step(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, int n, float lr, float b1, float b2, float eps,
                          float c1, float c2, float wd) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float gk = g[k] + wd * p[k];
  m[k] = b1 * m[k] + (1.f - b1) * gk;
  v[k] = b2 * v[k] + (1.f - b2) * gk * gk;
  p[k] -= lr * (m[k] / c1) / (sqrtf(v[k] / c2) + eps);
}

inline unsigned blocks(size_t n) { return (unsigned)((n + 255) / 256); }

// Device buffers of one forward/backward pass over n samples.
struct Pass {
  float *x = nullptr, *t = nullptr, *mask = nullptr, *h1 = nullptr, *h2 = nullptr, *y = nullptr;
  float *d3 = nullptr, *d2 = nullptr, *d1 = nullptr, *loss = nullptr;
};

// Forward pass; optionally the loss and the gradient (into g) as well.
void forward(const Dims& D, const float* p, const Pass& s, int n, cudaStream_t st) {
  linear_fwd<<<blocks((size_t)n * D.hidden), 256, 0, st>>>(s.x, p + D.w1(), p + D.b1(), s.h1, n,
                                                           D.in, D.hidden, 1);
  linear_fwd<<<blocks((size_t)n * D.hidden), 256, 0, st>>>(s.h1, p + D.w2(), p + D.b2(), s.h2, n,
                                                           D.hidden, D.hidden, 1);
  linear_fwd<<<blocks((size_t)n * D.out), 256, 0, st>>>(s.h2, p + D.w3(), p + D.b3(), s.y, n,
                                                        D.hidden, D.out, 0);
}

void backward(const Dims& D, const float* p, float* g, const Pass& s, int n, float inv_count,
              cudaStream_t st) {
  mse_grad<<<blocks((size_t)n * D.out), 256, 0, st>>>(s.y, s.t, s.mask, s.d3, n, D.out, inv_count,
                                                      s.loss);
  linear_bwd_w<<<blocks((size_t)D.out * (D.hidden + 1)), 256, 0, st>>>(s.d3, s.h2, g + D.w3(),
                                                                       g + D.b3(), n, D.hidden, D.out);
  linear_bwd_x<<<blocks((size_t)n * D.hidden), 256, 0, st>>>(s.d3, p + D.w3(), s.h2, s.d2, n,
                                                             D.hidden, D.out, 1);
  linear_bwd_w<<<blocks((size_t)D.hidden * (D.hidden + 1)), 256, 0, st>>>(s.d2, s.h1, g + D.w2(),
                                                                          g + D.b2(), n, D.hidden,
                                                                          D.hidden);
  linear_bwd_x<<<blocks((size_t)n * D.hidden), 256, 0, st>>>(s.d2, p + D.w2(), s.h1, s.d1, n,
                                                             D.hidden, D.hidden, 1);
  linear_bwd_w<<<blocks((size_t)D.hidden * (D.in + 1)), 256, 0, st>>>(s.d1, s.x, g + D.w1(),
                                                                      g + D.b1(), n, D.in, D.hidden);
}

struct DevMem {
  std::vector<void*> ptrs;
  ~DevMem() {
    for (void* p : ptrs) cudaFree(p);
  }
  cudaError_t alloc(float** p, size_t n) {
    cudaError_t e = cudaMalloc((void**)p, (n ? n : 1) * sizeof(float));
    if (e == cudaSuccess) ptrs.push_back(*p);
    return e;
  }
};

int alloc_pass(DevMem& mem, const Dims& D, int n, Pass* s) {
  SEL_CUDA(mem.alloc(&s->x, (size_t)n * D.in));
  SEL_CUDA(mem.alloc(&s->t, (size_t)n * D.out));
  SEL_CUDA(mem.alloc(&s->mask, (size_t)n * D.out));
  SEL_CUDA(mem.alloc(&s->h1, (size_t)n * D.hidden));
  SEL_CUDA(mem.alloc(&s->h2, (size_t)n * D.hidden));
  SEL_CUDA(mem.alloc(&s->y, (size_t)n * D.out));
  SEL_CUDA(mem.alloc(&s->d3, (size_t)n * D.out));
  SEL_CUDA(mem.alloc(&s->d2, (size_t)n * D.hidden));
  SEL_CUDA(mem.alloc(&s->d1, (size_t)n * D.hidden));
  SEL_CUDA(mem.alloc(&s->loss, 1));
  return ANB_OK;
}

int check_dims(int n, int in, int hidden, int out) {
  if (n <= 0 || in <= 0 || hidden <= 0 || out <= 0 || in > 4096 || hidden > 4096 || out > 4096)
    return sel_fail(ANB_ERR_ARG, "bad MLP dimensions");
  int dev = 0;
  if (cudaGetDeviceCount(&dev) != cudaSuccess || dev == 0)
    return sel_fail(ANB_ERR_CUDA, "no CUDA device is available");
  return ANB_OK;
}

}  // namespace

extern "C" {

const char* anb_selector_last_error(void) { return g_sel_error.c_str(); }

size_t anb_mlp_param_count(int in, int hidden, int out) {
  Dims D{in, hidden, out};
  return D.total();
}

int anb_mlp_loss_grad(const float* params, const float* x, const float* target, const float* mask,
                      int n, int in, int hidden, int out, float* loss, float* grad) {
  int rc = check_dims(n, in, hidden, out);
  if (rc) return rc;
  if (!params || !x || !target || !mask || !loss || !grad) return sel_fail(ANB_ERR_ARG, "NULL argument");
  Dims D{in, hidden, out};
  DevMem mem;
  Pass s;
  rc = alloc_pass(mem, D, n, &s);
  if (rc) return rc;
  float *p = nullptr, *g = nullptr;
  SEL_CUDA(mem.alloc(&p, D.total()));
  SEL_CUDA(mem.alloc(&g, D.total()));
  SEL_CUDA(cudaMemcpy(p, params, D.total() * sizeof(float), cudaMemcpyHostToDevice));
  SEL_CUDA(cudaMemcpy(s.x, x, (size_t)n * in * sizeof(float), cudaMemcpyHostToDevice));
  SEL_CUDA(cudaMemcpy(s.t, target, (size_t)n * out * sizeof(float), cudaMemcpyHostToDevice));
  SEL_CUDA(cudaMemcpy(s.mask, mask, (size_t)n * out * sizeof(float), cudaMemcpyHostToDevice));
  std::vector<float> hm((size_t)n * out);
  std::memcpy(hm.data(), mask, hm.size() * sizeof(float));
  double cnt = 0;
  for (float m : hm) cnt += m;
  const float inv = cnt > 0 ? (float)(1.0 / cnt) : 0.f;
  SEL_CUDA(cudaMemset(s.loss, 0, sizeof(float)));
  forward(D, p, s, n, 0);
  backward(D, p, g, s, n, inv, 0);
  SEL_CUDA(cudaGetLastError());
  SEL_CUDA(cudaMemcpy(loss, s.loss, sizeof(float), cudaMemcpyDeviceToHost));
  SEL_CUDA(cudaMemcpy(grad, g, D.total() * sizeof(float), cudaMemcpyDeviceToHost));
  return ANB_OK;
}

int anb_mlp_train(float* params, const float* x, const float* target, const float* mask, int n,
                  int in, int hidden, int out, int epochs, float lr, float weight_decay,
                  float* final_loss) {
  int rc = check_dims(n, in, hidden, out);
  if (rc) return rc;
  if (!params || !x || !target || !mask || epochs < 0) return sel_fail(ANB_ERR_ARG, "bad argument");
  Dims D{in, hidden, out};
  DevMem mem;
  Pass s;
  rc = alloc_pass(mem, D, n, &s);
  if (rc) return rc;
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  SEL_CUDA(mem.alloc(&p, D.total()));
  SEL_CUDA(mem.alloc(&g, D.total()));
  SEL_CUDA(mem.alloc(&m, D.total()));
  SEL_CUDA(mem.alloc(&v, D.total()));
  SEL_CUDA(cudaMemset(m, 0, D.total() * sizeof(float)));
  SEL_CUDA(cudaMemset(v, 0, D.total() * sizeof(float)));
  SEL_CUDA(cudaMemcpy(p, params, D.total() * sizeof(float), cudaMemcpyHostToDevice));
  SEL_CUDA(cudaMemcpy(s.x, x, (size_t)n * in * sizeof(float), cudaMemcpyHostToDevice));
  SEL_CUDA(cudaMemcpy(s.t, target, (size_t)n * out * sizeof(float), cudaMemcpyHostToDevice));
  SEL_CUDA(cudaMemcpy(s.mask, mask, (size_t)n * out * sizeof(float), cudaMemcpyHostToDevice));
  double cnt = 0;
  for (size_t k = 0; k < (size_t)n * out; ++k) cnt += mask[k];
  const float inv = cnt > 0 ? (float)(1.0 / cnt) : 0.f;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  double c1 = 1.0, c2 = 1.0;
  for (int e = 0; e < epochs; ++e) {
    SEL_CUDA(cudaMemsetAsync(s.loss, 0, sizeof(float), 0));
    forward(D, p, s, n, 0);
    backward(D, p, g, s, n, inv, 0);
    c1 *= b1;
    c2 *= b2;
    adam_step<<<blocks(D.total()), 256>>>(p, g, m, v, (int)D.total(), lr, b1, b2, eps,
                                          (float)(1.0 - c1), (float)(1.0 - c2), weight_decay);
  }
  SEL_CUDA(cudaGetLastError());
  SEL_CUDA(cudaDeviceSynchronize());
  if (final_loss) {
    SEL_CUDA(cudaMemsetAsync(s.loss, 0, sizeof(float), 0));
    forward(D, p, s, n, 0);
    mse_grad<<<blocks((size_t)n * D.out), 256>>>(s.y, s.t, s.mask, s.d3, n, D.out, inv, s.loss);
    SEL_CUDA(cudaMemcpy(final_loss, s.loss, sizeof(float), cudaMemcpyDeviceToHost));
  }
  SEL_CUDA(cudaMemcpy(params, p, D.total() * sizeof(float), cudaMemcpyDeviceToHost));
  return ANB_OK;
}

int anb_mlp_predict(const float* params, const float* x, int n, int in, int hidden, int out,
                    float* y) {
  int rc = check_dims(n, in, hidden, out);
  if (rc) return rc;
  if (!params || !x || !y) return sel_fail(ANB_ERR_ARG, "NULL argument");
  Dims D{in, hidden, out};
  DevMem mem;
  Pass s;
  float* p = nullptr;
  SEL_CUDA(mem.alloc(&p, D.total()));
  SEL_CUDA(mem.alloc(&s.x, (size_t)n * in));
  SEL_CUDA(mem.alloc(&s.h1, (size_t)n * hidden));
  SEL_CUDA(mem.alloc(&s.h2, (size_t)n * hidden));
  SEL_CUDA(mem.alloc(&s.y, (size_t)n * out));
  SEL_CUDA(cudaMemcpy(p, params, D.total() * sizeof(float), cudaMemcpyHostToDevice));
  SEL_CUDA(cudaMemcpy(s.x, x, (size_t)n * in * sizeof(float), cudaMemcpyHostToDevice));
  forward(D, p, s, n, 0);
  SEL_CUDA(cudaGetLastError());
  SEL_CUDA(cudaMemcpy(y, s.y, (size_t)n * out * sizeof(float), cudaMemcpyDeviceToHost));
  return ANB_OK;
}

}  // extern "C"

// ---- forward pass without allocation ------------------------------------
//
// anb_mlp_predict above allocates device buffers on every call. Some callers
// cannot do that: a simulation loop with real-time deadlines, where the
// implicit device synchronisation of cudaMalloc/cudaFree would stall it, and
// host programs whose device memory is owned by another allocator (a memory
// pool or a framework's caching allocator) that forbids allocations outside
// it. They pass device buffers they already own for the parameters, the
// inputs and the outputs; the two hidden-layer activations go to the fixed
// array below instead of freshly allocated memory.
//
// The array is part of this library's device image: every GPU that loads the
// library holds it (2 MiB) until the process exits. All calls share it and it
// keeps the last call's contents; the forward pass overwrites every element
// it reads, so nothing needs clearing. Calls whose work overlaps on the GPU
// (different streams, or different host threads on one device) race on it.

constexpr size_t kNoAllocScratchFloats = (size_t)1 << 19;  // 2 MiB of float
static __device__ __align__(256) float anb_mlp_noalloc_scratch[kNoAllocScratchFloats];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
float* g_noalloc_ptr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device. In host code
// the array's name only stands for the symbol; the address must come from
// cudaGetSymbolAddress, once per device, with that device current.
int noalloc_scratch(float** out) {
  int dev = 0;
  SEL_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return sel_fail(ANB_ERR_ARG, "device index out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, anb_mlp_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return sel_fail(ANB_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") +
                                        cudaGetErrorString(e));
    g_noalloc_ptr[dev] = static_cast<float*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return ANB_OK;
}

}  // namespace

extern "C" {

size_t anb_mlp_noalloc_max_floats(void) { return kNoAllocScratchFloats; }

int anb_mlp_predict_noalloc(const float* params, const float* x, int n, int in, int hidden, int out,
                            float* y, void* stream) {
  int rc = check_dims(n, in, hidden, out);
  if (rc) return rc;
  if (!params || !x || !y) return sel_fail(ANB_ERR_ARG, "NULL argument");
  const size_t need = 2 * (size_t)n * (size_t)hidden;
  if (need > kNoAllocScratchFloats)
    return sel_fail(ANB_ERR_ARG, "anb_mlp_predict_noalloc: n * hidden = " +
                                     std::to_string((size_t)n * hidden) + " exceeds the limit of " +
                                     std::to_string(kNoAllocScratchFloats / 2) +
                                     " activations per layer");
  float* scratch = nullptr;
  rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  Dims D{in, hidden, out};
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  float* h1 = scratch;
  float* h2 = scratch + (size_t)n * hidden;
  linear_fwd<<<blocks((size_t)n * D.hidden), 256, 0, st>>>(x, params + D.w1(), params + D.b1(), h1,
                                                           n, D.in, D.hidden, 1);
  linear_fwd<<<blocks((size_t)n * D.hidden), 256, 0, st>>>(h1, params + D.w2(), params + D.b2(),
                                                           h2, n, D.hidden, D.hidden, 1);
  linear_fwd<<<blocks((size_t)n * D.out), 256, 0, st>>>(h2, params + D.w3(), params + D.b3(), y, n,
                                                        D.hidden, D.out, 0);
  SEL_CUDA(cudaGetLastError());
  return ANB_OK;
}

}  // extern "C"
