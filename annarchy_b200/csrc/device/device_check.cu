// Build-time instantiation of every device template of anb_device.cuh with
// the types the code generator uses, compiled by nvcc for sm_100a. The
// generated network modules are compiled by NVRTC at run time; this file
// makes the build fail early if the header stops compiling, and its
// -Xptxas -v output reports registers and spills of each template.
#include "anb_device.cuh"

extern "C" __global__ void check_rate_csr_scalar(int n, const int* rp, const int* c, const double* w,
                                                 const double* r, const int* pr, double* s) {
  anb_rate_csr_scalar<double, double, int>(n, rp, c, w, r, pr, s);
  anb_rate_csr_ordered<double, double, int>(n, rp, c, w, r, pr, s);
}
extern "C" __global__ void check_rate_csr_delayed(int n, const int* rp, const int* c, const double* w,
                                                  const int* d, const double* ring, int n_pre, int slots,
                                                  long long t, const int* pr, double* s) {
  anb_rate_csr_delayed_ordered<double, double, int>(n, rp, c, w, d, ring, n_pre, slots, t, pr, s);
  anb_rate_csr_delayed_ordered<float, float, int>(n, rp, c, reinterpret_cast<const float*>(w), d,
                                                  reinterpret_cast<const float*>(ring), n_pre, slots, t, pr,
                                                  reinterpret_cast<float*>(s));
}
extern "C" __global__ void check_rate_csr_vector_f32(int n, const int* rp, const int* c, const float* w,
                                                     const float* r, const int* pr, float* s) {
  anb_rate_csr_vector<8, float, int>(n, rp, c, w, r, pr, s, 10000);
}
extern "C" __global__ void check_rate_csr_vector_bf16(int n, const int* rp, const int* c,
                                                      const anb_bf16* w, const float* r, const int* pr,
                                                      float* s) {
  anb_rate_csr_vector<32, anb_bf16, int>(n, rp, c, w, r, pr, s, 10000);
}
extern "C" __global__ void check_rate_ell(int n, int width, const int* c, const float* w, const int* rl,
                                          const float* r, const int* pr, float* s) {
  anb_rate_ell<float, float>(n, width, c, w, rl, r, pr, s);
}
extern "C" __global__ void check_rate_sell(int n, const int* sp, const int* sl, const int* c,
                                           const anb_bf16* w, const int* rl, const int* perm,
                                           const float* r, const int* pr, float* s) {
  anb_rate_sell<32, float, anb_bf16>(n, sp, sl, c, w, rl, perm, r, pr, s);
}
extern "C" __global__ void check_spike_gather(int n, const int* rp, const int* c, const double* w,
                                              const anb_u32* spk, const int* pr, double* g) {
  anb_spike_gather<double, double>(n, rp, c, w, spk, pr, g);
}
extern "C" __global__ void check_spike_scatter(const anb_u32* spk, const int* cp, const int* pi,
                                               const anb_bf16* w, float* g) {
  anb_spike_scatter<float, anb_bf16>(0, 128, spk, cp, pi, w, g);
}
extern "C" __global__ void __launch_bounds__(384, 3) check_rate_pcsr_f32(
    const int* cp, const int* wt, const unsigned short* c, const float* w, const float* x, int n_pre,
    int pw, float* s, int* err) {
  anb_rate_pcsr<float, 8>(cp, wt, c, w, x, n_pre, pw, s, err);
}
extern "C" __global__ void __launch_bounds__(384, 3) check_rate_pcsr_bf16(
    const int* cp, const int* wt, const unsigned short* c, const anb_bf16* w, const float* x, int n_pre,
    int pw, float* s, int* err) {
  anb_rate_pcsr<anb_bf16, 8>(cp, wt, c, w, x, n_pre, pw, s, err);
}
