// Device-side building blocks shared by every generated network module.
//
// The generated source (annarchy_b200/generator/codegen.py) includes this
// text first, then declares one __constant__ pointer per device array
// (bound by the runtime) and the network's kernels, which call the
// templates below. Compiled by NVRTC for sm_100a.
//
// Numerics: the double-precision ("exact") kernels keep the reference's
// operation order — one sequential sum per row in ascending pre rank,
// conductance increments applied per post neuron in ascending pre rank —
// and the module is compiled without multiply-add contraction, so results
// are bit-identical to the reference CPU build compiled with
// -ffp-contract=off. The single-precision ("fast") kernels reorder sums
// freely (atomics, vector loads) and are checked against tolerances.
#pragma once

typedef unsigned int anb_u32;
typedef unsigned short anb_bf16;   // bfloat16 storage (upper half of an IEEE float)
typedef long long anb_i64;

#define ANB_WARP 32

// Error codes a kernel writes into the network's error word.
#ifndef M_PI
#define M_PI 3.14159265358979323846   // pi in equations (the reference's sympy output)
#endif
#define ANB_DEVERR_BARRIER_TIMEOUT 1
#define ANB_DEVERR_INDEX 2
#define ANB_DEVERR_MONITOR_OVERFLOW 3

// ---- built-in functions of the equation language --------------------------
// (names as emitted by the reference parser: ANNarchy/parser/ParserTemplate.py)
template <typename T> __device__ __forceinline__ T positive(T x) { return x > T(0) ? x : T(0); }
template <typename T> __device__ __forceinline__ T negative(T x) { return x < T(0) ? x : T(0); }
// modulo(a, b): the integer remainder of a and b truncated to 64-bit
// integers (the reference's `long(a) % long(b)`)
template <typename A, typename B>
__device__ __forceinline__ long long modulo(A a, B b) { return (long long)a % (long long)b; }
// power(x, a): x multiplied by itself, a converted to an unsigned integer
// exponent (the reference's integer power, a - 1 multiplications in order);
// an exponent of 0 gives x
__device__ __forceinline__ double power(double x, unsigned int a) {
  double r = x;
  for (unsigned int i = 1; i < a; ++i) r *= x;
  return r;
}
__device__ __forceinline__ float power(float x, unsigned int a) {
  float r = x;
  for (unsigned int i = 1; i < a; ++i) r *= x;
  return r;
}
__device__ __forceinline__ double power(int x, unsigned int a) { return power((double)x, a); }
#define clip(x, a, b) ((x) < (a) ? (a) : ((x) > (b) ? (b) : (x)))
#define ite(a, b, c) ((a) ? (b) : (c))

// ---- bfloat16 ---------------------------------------------------------------
__device__ __forceinline__ float anb_bf16_to_f32(anb_bf16 h) {
  return __uint_as_float(((anb_u32)h) << 16);
}
// Weight value in arithmetic precision: doubles stay double, floats float,
// bfloat16 is widened to float.
__device__ __forceinline__ double anb_wf(double w) { return w; }
__device__ __forceinline__ float anb_wf(float w) { return w; }
__device__ __forceinline__ float anb_wf(anb_bf16 w) { return anb_bf16_to_f32(w); }

// ---- spike bitmaps -------------------------------------------------------------
__device__ __forceinline__ bool anb_bit(const anb_u32* bits, int i) {
  return (bits[i >> 5] >> (i & 31)) & 1u;
}

// Start of every kernel of the grid engine's plan, which may be launched
// while the previous kernel of the stream still runs (programmatic dependent
// launch): wait until that kernel has finished and its writes are visible,
// then allow the next kernel to be scheduled. Outside such a launch both
// return at once.
__device__ __forceinline__ void anb_pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ void anb_report(int* err, int code) {
  if (err) atomicCAS(err, 0, code);
}

// ---- rate-coded weighted sums ------------------------------------------------------

// Thread per row, sequential sum in stored (ascending pre) order:
// sum[post_rank[row]] += sum_j w[j] * r[col[j]]  (double, reference order).
template <typename R, typename W, typename I>
__device__ __forceinline__ void anb_rate_csr_scalar(int n_rows, const I* __restrict__ row_ptr,
                                                    const int* __restrict__ col,
                                                    const W* __restrict__ w,
                                                    const R* __restrict__ pre_r,
                                                    const int* __restrict__ post_rank,
                                                    R* __restrict__ sum) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n_rows;
       row += gridDim.x * blockDim.x) {
    R s = R(0);
    const I beg = row_ptr[row], end = row_ptr[row + 1];
    for (I j = beg; j < end; ++j) s += pre_r[col[j]] * (R)w[j];
    const int post = post_rank ? post_rank[row] : row;
    sum[post] += s;
  }
}

// Warp per row, the same sum in the same order as anb_rate_csr_scalar: the
// lanes form 32 products pre_r[col[j]] * w[j] at a time (coalesced index and
// weight loads, all gathers in flight, the next 32 loading while these are
// added), then every lane adds them one by one in stored order, as the
// reference's sequential loop does (ANNarchy/generator/Projection/OpenMP/
// CSR.py:177-253); no addition is reordered, so the result is the scalar
// kernel's bit for bit.
template <typename R, typename W, typename I>
__device__ __forceinline__ void anb_rate_csr_ordered(int n_rows, const I* __restrict__ row_ptr,
                                                     const int* __restrict__ col,
                                                     const W* __restrict__ w,
                                                     const R* __restrict__ pre_r,
                                                     const int* __restrict__ post_rank,
                                                     R* __restrict__ sum) {
  const int lane = threadIdx.x & 31;
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  for (int row = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); row < n_rows; row += nwarps) {
    const I beg = row_ptr[row], end = row_ptr[row + 1];
    R s = R(0);
    I j = beg + lane;
    R p = j < end ? pre_r[col[j]] * (R)w[j] : R(0);
    for (I j0 = beg; j0 < end; j0 += 32) {
      const I jn = j0 + 32 + lane;
      const R pn = jn < end ? pre_r[col[jn]] * (R)w[jn] : R(0);
      if (end - j0 >= 32) {
#pragma unroll
        for (int k = 0; k < 32; ++k) s += __shfl_sync(0xffffffffu, p, k);
      } else {
        const int cnt = (int)(end - j0);
        for (int k = 0; k < cnt; ++k) s += __shfl_sync(0xffffffffu, p, k);
      }
      p = pn;
    }
    if (lane == 0) sum[post_rank ? post_rank[row] : row] += s;
  }
}

// ---- random numbers in equations --------------------------------------------------------
// Counter-based generator Philox4x32-10 (J. K. Salmon, M. A. Moraes, R. O. Dror,
// D. E. Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11): ten
// rounds of two 32x32->64 multiplications with the published multipliers
// and Weyl key increments. A draw is a pure function of (seed, stream,
// step, neuron), so no generator state is stored or advanced, and every
// neuron of every step draws independently in any launch order.
struct anb_u4 {
  unsigned x, y, z, w;
};

__device__ __forceinline__ anb_u4 anb_philox4x32_10(anb_u4 c, unsigned k0, unsigned k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const unsigned long long p0 = (unsigned long long)0xD2511F53u * c.x;
    const unsigned long long p1 = (unsigned long long)0xCD9E8D57u * c.z;
    const unsigned hi0 = (unsigned)(p0 >> 32), lo0 = (unsigned)p0;
    const unsigned hi1 = (unsigned)(p1 >> 32), lo1 = (unsigned)p1;
    c = anb_u4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// The four 32-bit words of draw (seed, stream, step t, index i).
__device__ __forceinline__ anb_u4 anb_rand_words(const unsigned* seed, unsigned stream, long long t,
                                                 unsigned i) {
  return anb_philox4x32_10(anb_u4{i, (unsigned)t, (unsigned)((unsigned long long)t >> 32), stream},
                           seed[0], seed[1]);
}

// Uniform on [0, 1): 24 bits (float) or 53 bits (double) of the first words.
template <typename R>
__device__ __forceinline__ R anb_unit(const anb_u4& w);
template <>
__device__ __forceinline__ float anb_unit<float>(const anb_u4& w) {
  return (float)(w.x >> 8) * (1.0f / 16777216.0f);
}
template <>
__device__ __forceinline__ double anb_unit<double>(const anb_u4& w) {
  return (double)(((unsigned long long)(w.x >> 6) << 27) | (w.y >> 5)) * (1.0 / 9007199254740992.0);
}

// Standard normal by the Box-Muller transform of two uniforms (the second
// pair of words); u1 in (0, 1] keeps the logarithm finite.
template <typename R>
__device__ __forceinline__ R anb_std_normal(const anb_u4& w) {
  const anb_u4 v{w.z, w.w, w.x, w.y};
  const R u1 = R(1) - anb_unit<R>(w), u2 = anb_unit<R>(v);
  return sqrt(R(-2) * log(u1)) * cos(R(6.283185307179586) * u2);
}

template <typename R>
__device__ __forceinline__ R anb_draw_uniform(const unsigned* seed, unsigned stream, long long t,
                                              unsigned i, R lo, R hi) {
  return lo + (hi - lo) * anb_unit<R>(anb_rand_words(seed, stream, t, i));
}
template <typename R>
__device__ __forceinline__ R anb_draw_normal(const unsigned* seed, unsigned stream, long long t,
                                             unsigned i, R mu, R sigma) {
  return mu + sigma * anb_std_normal<R>(anb_rand_words(seed, stream, t, i));
}
template <typename R>
__device__ __forceinline__ R anb_draw_lognormal(const unsigned* seed, unsigned stream, long long t,
                                                unsigned i, R mu, R sigma) {
  return exp(mu + sigma * anb_std_normal<R>(anb_rand_words(seed, stream, t, i)));
}
template <typename R>
__device__ __forceinline__ R anb_draw_exponential(const unsigned* seed, unsigned stream, long long t,
                                                  unsigned i, R lambda) {
  return -log(R(1) - anb_unit<R>(anb_rand_words(seed, stream, t, i))) / lambda;
}
template <typename R>
__device__ __forceinline__ R anb_draw_discrete_uniform(const unsigned* seed, unsigned stream, long long t,
                                                       unsigned i, R lo, R hi) {
  return lo + floor(anb_unit<R>(anb_rand_words(seed, stream, t, i)) * (hi - lo + R(1)));
}

// Slot of time step s (possibly negative) in a ring of `slots` entries.
__device__ __forceinline__ int anb_ring_slot(long long s, int slots) {
  const long long m = s % slots;
  return (int)(m < 0 ? m + slots : m);
}

// Rate-coded weighted sum with one transmission delay per synapse (steps,
// >= 1): thread per row, sequential in stored order like anb_rate_csr_scalar,
// each rate read from the pre population's history ring (slot of step
// t - delay; slots x n_pre values). The reference's non-uniform delays read
// pre.r from its queue entry delay - 1 (ANNarchy/generator/Projection/
// SingleThreadGenerator.py, _computesum_rate with max_delay > 1).
// The same sum with a warp per row (products gathered 32 at a time, added
// one by one in stored order, as anb_rate_csr_ordered).
template <typename R, typename W, typename I>
__device__ __forceinline__ void anb_rate_csr_delayed_ordered(int n_rows, const I* __restrict__ row_ptr,
                                                             const int* __restrict__ col,
                                                             const W* __restrict__ w,
                                                             const int* __restrict__ dly,
                                                             const R* __restrict__ ring, int n_pre,
                                                             int slots, long long t,
                                                             const int* __restrict__ post_rank,
                                                             R* __restrict__ sum) {
  const int lane = threadIdx.x & 31;
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  for (int row = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); row < n_rows; row += nwarps) {
    const I beg = row_ptr[row], end = row_ptr[row + 1];
    R s = R(0);
    I j = beg + lane;
    R p = j < end ? ring[(size_t)anb_ring_slot(t - dly[j], slots) * n_pre + col[j]] * (R)w[j] : R(0);
    for (I j0 = beg; j0 < end; j0 += 32) {
      const I jn = j0 + 32 + lane;
      const R pn = jn < end ? ring[(size_t)anb_ring_slot(t - dly[jn], slots) * n_pre + col[jn]] * (R)w[jn]
                            : R(0);
      const int cnt = end - j0 >= 32 ? 32 : (int)(end - j0);
      for (int k = 0; k < cnt; ++k) s += __shfl_sync(0xffffffffu, p, k);
      p = pn;
    }
    if (lane == 0) sum[post_rank ? post_rank[row] : row] += s;
  }
}

template <typename R, typename W, typename I>
__device__ __forceinline__ void anb_rate_csr_delayed(int n_rows, const I* __restrict__ row_ptr,
                                                     const int* __restrict__ col,
                                                     const W* __restrict__ w,
                                                     const int* __restrict__ dly,
                                                     const R* __restrict__ ring, int n_pre,
                                                     int slots, long long t,
                                                     const int* __restrict__ post_rank,
                                                     R* __restrict__ sum) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n_rows;
       row += gridDim.x * blockDim.x) {
    R s = R(0);
    const I beg = row_ptr[row], end = row_ptr[row + 1];
    for (I j = beg; j < end; ++j)
      s += ring[(size_t)anb_ring_slot(t - dly[j], slots) * n_pre + col[j]] * (R)w[j];
    const int post = post_rank ? post_rank[row] : row;
    sum[post] += s;
  }
}

// Sub-warp per row (G lanes, G in {2,4,8,16,32}), fp32 accumulation with a
// butterfly reduction. Rows longer than `kahan_min` use compensated
// (Kahan) summation per lane.
template <int G, typename W, typename I>
__device__ __forceinline__ void anb_rate_csr_vector(int n_rows, const I* __restrict__ row_ptr,
                                                    const int* __restrict__ col,
                                                    const W* __restrict__ w,
                                                    const float* __restrict__ pre_r,
                                                    const int* __restrict__ post_rank,
                                                    float* __restrict__ sum, int kahan_min) {
  const int lane = threadIdx.x % G;
  const int groups = (gridDim.x * blockDim.x) / G;
  for (int row = (blockIdx.x * blockDim.x + threadIdx.x) / G; row < n_rows; row += groups) {
    const I beg = row_ptr[row], end = row_ptr[row + 1];
    float s = 0.f;
    if (end - beg >= (I)kahan_min) {
      float c = 0.f;
      for (I j = beg + lane; j < end; j += G) {
        float y = __fmul_rn(__ldg(&pre_r[__ldg(&col[j])]), anb_wf(w[j])) - c;
        float t = s + y;
        c = (t - s) - y;
        s = t;
      }
    } else {
      for (I j = beg + lane; j < end; j += G) s += __ldg(&pre_r[__ldg(&col[j])]) * anb_wf(w[j]);
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, G);
    if (lane == 0) {
      const int post = post_rank ? post_rank[row] : row;
      sum[post] += s;
    }
  }
}

// Streaming loads of matrix data that is read once per step: not allocated
// in L1, so L1 keeps the gathered pre-synaptic vector.
__device__ __forceinline__ int4 anb_ls_i4(const int4* p) {
  int4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.s32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p));
  return v;
}
__device__ __forceinline__ float4 anb_ls_f4(const float4* p) {
  float4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
  return v;
}
__device__ __forceinline__ uint2 anb_ls_u2(const uint2* p) {
  uint2 v;
  asm volatile("ld.global.nc.L1::no_allocate.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "l"(p));
  return v;
}
__device__ __forceinline__ int anb_ls_i(const int* p) {
  int v;
  asm volatile("ld.global.nc.L1::no_allocate.s32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ float anb_ls_f(const float* p) {
  float v;
  asm volatile("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ unsigned short anb_ls_h(const unsigned short* p) {
  unsigned short v;
  asm volatile("ld.global.nc.L1::no_allocate.u16 %0, [%1];" : "=h"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ uint4 anb_ls_u4(const uint4* p) {
  uint4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p));
  return v;
}
__device__ __forceinline__ anb_u32 anb_ls_u(const anb_u32* p) {
  anb_u32 v;
  asm volatile("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

// Bulk prefetch of a byte range of global memory into L2; the address and
// the size are multiples of 16 bytes and the range lies inside one array.
__device__ __forceinline__ void anb_prefetch_l2(const void* p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(p), "r"(bytes) : "memory");
}

// Four consecutive weights widened to float (16-byte or 8-byte load).
__device__ __forceinline__ float4 anb_w4(const float* w) { return anb_ls_f4(reinterpret_cast<const float4*>(w)); }
__device__ __forceinline__ float4 anb_w4(const anb_bf16* w) {
  const uint2 u = anb_ls_u2(reinterpret_cast<const uint2*>(w));
  return make_float4(__uint_as_float(u.x << 16), __uint_as_float(u.x & 0xffff0000u),
                     __uint_as_float(u.y << 16), __uint_as_float(u.y & 0xffff0000u));
}
__device__ __forceinline__ float anb_w1(const float* w) { return anb_ls_f(w); }
__device__ __forceinline__ float anb_w1(const anb_bf16* w) { return anb_bf16_to_f32(anb_ls_h(w)); }

// Sub-warp per row with 16-byte vector loads of the column indices and
// weights (streaming, evict-first) over the 4-aligned body of every row and
// scalar loads at its ends. `rows` (optional) lists the rows to process
// (row-length binning); `n_rows` is its length.
template <int G, typename W>
__device__ __forceinline__ void anb_rate_csr_vec(int n_rows, const int* __restrict__ rows,
                                                 const int* __restrict__ row_ptr,
                                                 const int* __restrict__ col,
                                                 const W* __restrict__ w,
                                                 const float* __restrict__ x,
                                                 const int* __restrict__ post_rank,
                                                 float* __restrict__ sum) {
  const int lane = threadIdx.x % G;
  const int groups = (gridDim.x * blockDim.x) / G;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) / G; r < n_rows; r += groups) {
    const int row = rows ? rows[r] : r;
    const int beg = row_ptr[row], end = row_ptr[row + 1];
    int j0 = (beg + 3) & ~3;
    if (j0 > end) j0 = end;
    float s = 0.f;
    for (int j = beg + lane; j < j0; j += G) s += __ldg(&x[anb_ls_i(&col[j])]) * anb_w1(&w[j]);
    const int nv = (end - j0) >> 2;
    const int4* __restrict__ c4 = reinterpret_cast<const int4*>(col + j0);
    float s1 = 0.f;
    int v = lane;
    for (; v + G < nv; v += 2 * G) {          // two vectors in flight per lane
      const int4 ca = anb_ls_i4(c4 + v), cb = anb_ls_i4(c4 + v + G);
      const float4 wa = anb_w4(w + j0 + 4 * v), wb = anb_w4(w + j0 + 4 * (v + G));
      s += __ldg(&x[ca.x]) * wa.x + __ldg(&x[ca.y]) * wa.y + __ldg(&x[ca.z]) * wa.z +
           __ldg(&x[ca.w]) * wa.w;
      s1 += __ldg(&x[cb.x]) * wb.x + __ldg(&x[cb.y]) * wb.y + __ldg(&x[cb.z]) * wb.z +
            __ldg(&x[cb.w]) * wb.w;
    }
    if (v < nv) {
      const int4 c = anb_ls_i4(c4 + v);
      const float4 ww = anb_w4(w + j0 + 4 * v);
      s += __ldg(&x[c.x]) * ww.x + __ldg(&x[c.y]) * ww.y + __ldg(&x[c.z]) * ww.z +
           __ldg(&x[c.w]) * ww.w;
    }
    s += s1;
    for (int j = j0 + 4 * nv + lane; j < end; j += G) s += __ldg(&x[anb_ls_i(&col[j])]) * anb_w1(&w[j]);
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, G);
    if (lane == 0) sum[post_rank ? post_rank[row] : row] += s;
  }
}

// One CTA per (long) row, Kahan-compensated per thread, block reduction.
template <typename W>
__device__ __forceinline__ void anb_rate_csr_cta(int n_rows, const int* __restrict__ rows,
                                                 const int* __restrict__ row_ptr,
                                                 const int* __restrict__ col,
                                                 const W* __restrict__ w,
                                                 const float* __restrict__ x,
                                                 const int* __restrict__ post_rank,
                                                 float* __restrict__ sum) {
  __shared__ float red[32];
  for (int r = blockIdx.x; r < n_rows; r += gridDim.x) {
    const int row = rows ? rows[r] : r;
    const int beg = row_ptr[row], end = row_ptr[row + 1];
    float s = 0.f, c = 0.f;
    for (int j = beg + threadIdx.x; j < end; j += blockDim.x) {
      const float y = __fmul_rn(__ldg(&x[anb_ls_i(&col[j])]), anb_w1(&w[j])) - c;
      const float t = s + y;
      c = (t - s) - y;
      s = t;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
      float v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (threadIdx.x == 0) sum[post_rank ? post_rank[row] : row] += v;
    }
    __syncthreads();
  }
}

// Blocked CSR with T x T tiles stored column-major (val[tile][c][r]): one
// CTA per block row; thread (r, part) sums tile row r over its share of the
// tile columns, then the parts are added in shared memory. Exact mode keeps
// one part per row (ascending columns = ascending pre rank).
template <int T, int PARTS, typename R, typename W>
__device__ __forceinline__ void anb_rate_bsr_rows(int n_block_rows, const int* __restrict__ brow_ptr,
                                                  const int* __restrict__ bcol,
                                                  const W* __restrict__ val,
                                                  const R* __restrict__ x, int n_pre, int n_post,
                                                  R* __restrict__ sum) {
  __shared__ R part[PARTS][T];
  const int r = threadIdx.x % T, pidx = threadIdx.x / T;
  constexpr int CW = T / PARTS;
  for (int br = blockIdx.x; br < n_block_rows; br += gridDim.x) {
    R s = R(0);
    if (pidx < PARTS) {
      for (int b = brow_ptr[br]; b < brow_ptr[br + 1]; ++b) {
        const W* __restrict__ tile = val + (size_t)b * T * T;
        const int c0 = bcol[b] * T;
        const R* __restrict__ xs = x + c0;
        const int cend = min((pidx + 1) * CW, n_pre - c0);   // partial last tile column
        for (int c = pidx * CW; c < cend; ++c) s += xs[c] * (R)anb_wf(tile[c * T + r]);
      }
      part[pidx][r] = s;
    }
    __syncthreads();
    if (pidx == 0) {
      R tot = part[0][r];
      for (int q = 1; q < PARTS; ++q) tot += part[q][r];
      const int post = br * T + r;
      if (post < n_post) sum[post] += tot;
    }
    __syncthreads();
  }
}

// ELLPACK / ELLPACK-R: column-major slots, thread per row.
// cols[k*n_rows + row], w likewise; rl = row lengths (ELL-R) or nullptr
// (ELL: stop at the first slot holding -1).
template <typename R, typename W>
__device__ __forceinline__ void anb_rate_ell(int n_rows, int width, const int* __restrict__ cols,
                                             const W* __restrict__ w, const int* __restrict__ rl,
                                             const R* __restrict__ pre_r,
                                             const int* __restrict__ post_rank,
                                             R* __restrict__ sum) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n_rows;
       row += gridDim.x * blockDim.x) {
    const int len = rl ? rl[row] : width;
    R s = R(0);
    if (sizeof(R) == 8 || !rl) {
      // exact order (double) or ELL with -1 padding: one chain
      for (int k = 0; k < len; ++k) {
        const int c = cols[(size_t)k * n_rows + row];
        if (!rl && c < 0) break;
        s += pre_r[c] * (R)anb_wf(w[(size_t)k * n_rows + row]);
      }
    } else {
      // four independent chains keep four gathers in flight per thread
      R s1 = R(0), s2 = R(0), s3 = R(0);
      int k = 0;
      for (; k + 4 <= len; k += 4) {
        const size_t o = (size_t)k * n_rows + row;
        const int c0 = __ldcs(&cols[o]), c1 = __ldcs(&cols[o + n_rows]);
        const int c2 = __ldcs(&cols[o + 2 * (size_t)n_rows]), c3 = __ldcs(&cols[o + 3 * (size_t)n_rows]);
        const R w0 = (R)anb_wf(w[o]), w1 = (R)anb_wf(w[o + n_rows]);
        const R w2 = (R)anb_wf(w[o + 2 * (size_t)n_rows]), w3 = (R)anb_wf(w[o + 3 * (size_t)n_rows]);
        s += __ldg(&pre_r[c0]) * w0;
        s1 += __ldg(&pre_r[c1]) * w1;
        s2 += __ldg(&pre_r[c2]) * w2;
        s3 += __ldg(&pre_r[c3]) * w3;
      }
      for (; k < len; ++k) {
        const size_t o = (size_t)k * n_rows + row;
        s += __ldg(&pre_r[__ldcs(&cols[o])]) * (R)anb_wf(w[o]);
      }
      s = (s + s1) + (s2 + s3);
    }
    const int post = post_rank ? post_rank[row] : row;
    sum[post] += s;
  }
}

// ELL / ELL-R / SELL in single precision with G threads per row: a CTA of
// R*G threads covers R consecutive rows (consecutive lanes = consecutive rows,
// so every load instruction is one contiguous run); thread part g takes slots
// g, g+G, ...; the G partial sums are added in shared memory.
// SELL passes its slice layout (slot of (row, k) = slice_ptr[row/C] + k*C + row%C);
// ELL passes slice_ptr = nullptr (slot = k*n_rows + row).
template <int G, int C, typename W>
__device__ __forceinline__ void anb_rate_slots_split(int n_rows, int width,
                                                     const int* __restrict__ slice_ptr,
                                                     const int* __restrict__ cols,
                                                     const W* __restrict__ w,
                                                     const int* __restrict__ rl,
                                                     const int* __restrict__ perm,
                                                     const float* __restrict__ x,
                                                     const int* __restrict__ post_rank,
                                                     float* __restrict__ sum) {
  __shared__ float part[1024];
  const int R = blockDim.x / G;
  const int lr = threadIdx.x % R, g = threadIdx.x / R;
  for (int base = blockIdx.x * R; base < n_rows; base += gridDim.x * R) {
    const int r = base + lr;
    float s = 0.f, s1 = 0.f;
    if (r < n_rows) {
      const int len = rl ? rl[r] : width;
      size_t slot0, stride;
      if (slice_ptr) {
        slot0 = (size_t)slice_ptr[r / C] + (r % C);
        stride = C;
      } else {
        slot0 = r;
        stride = (size_t)n_rows;
      }
      int k = g;
      for (; k + G < len; k += 2 * G) {
        const size_t o0 = slot0 + (size_t)k * stride, o1 = o0 + (size_t)G * stride;
        const int c0 = anb_ls_i(&cols[o0]), c1 = anb_ls_i(&cols[o1]);
        if (!rl && c1 < 0) {
          if (c0 >= 0) s += __ldg(&x[c0]) * anb_w1(&w[o0]);
          k = len;
          break;
        }
        s += __ldg(&x[c0]) * anb_w1(&w[o0]);
        s1 += __ldg(&x[c1]) * anb_w1(&w[o1]);
      }
      if (k < len) {
        const size_t o0 = slot0 + (size_t)k * stride;
        const int c0 = anb_ls_i(&cols[o0]);
        if (rl || c0 >= 0) s += __ldg(&x[c0]) * anb_w1(&w[o0]);
      }
    }
    part[threadIdx.x] = s + s1;
    __syncthreads();
    if (g == 0 && r < n_rows) {
      float tot = part[lr];
      for (int q = 1; q < G; ++q) tot += part[lr + q * R];
      const int row = perm ? perm[r] : r;
      sum[post_rank ? post_rank[row] : row] += tot;
    }
    __syncthreads();
  }
}

// SELL-C-sigma: slices of C consecutive (sorted) rows, column-major inside
// a slice; slice_ptr[s] = first slot of slice s, slice_len[s] = its width.
// perm[row in slice order] = original row. Thread per row.
template <int C, typename R, typename W>
__device__ __forceinline__ void anb_rate_sell(int n_rows, const int* __restrict__ slice_ptr,
                                              const int* __restrict__ slice_len,
                                              const int* __restrict__ cols,
                                              const W* __restrict__ w,
                                              const int* __restrict__ row_len,
                                              const int* __restrict__ perm,
                                              const R* __restrict__ pre_r,
                                              const int* __restrict__ post_rank,
                                              R* __restrict__ sum) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n_rows; r += gridDim.x * blockDim.x) {
    const int sl = r / C, lane = r % C;
    const int base = slice_ptr[sl];
    const int len = row_len[r];
    R s = R(0);
    if (sizeof(R) == 8) {
      for (int k = 0; k < len; ++k) {
        const int slot = base + k * C + lane;
        s += pre_r[cols[slot]] * (R)anb_wf(w[slot]);
      }
    } else {
      R s1 = R(0), s2 = R(0), s3 = R(0);
      int k = 0;
      for (; k + 4 <= len; k += 4) {
        const int o = base + k * C + lane;
        const int c0 = __ldcs(&cols[o]), c1 = __ldcs(&cols[o + C]);
        const int c2 = __ldcs(&cols[o + 2 * C]), c3 = __ldcs(&cols[o + 3 * C]);
        const R w0 = (R)anb_wf(w[o]), w1 = (R)anb_wf(w[o + C]);
        const R w2 = (R)anb_wf(w[o + 2 * C]), w3 = (R)anb_wf(w[o + 3 * C]);
        s += __ldg(&pre_r[c0]) * w0;
        s1 += __ldg(&pre_r[c1]) * w1;
        s2 += __ldg(&pre_r[c2]) * w2;
        s3 += __ldg(&pre_r[c3]) * w3;
      }
      for (; k < len; ++k) {
        const int o = base + k * C + lane;
        s += __ldg(&pre_r[__ldcs(&cols[o])]) * (R)anb_wf(w[o]);
      }
      s = (s + s1) + (s2 + s3);
    }
    const int row = perm ? perm[r] : r;
    const int post = post_rank ? post_rank[row] : row;
    sum[post] += s;
  }
}

// COO tail of HYB: one thread per entry, atomic accumulation (fast mode) —
// the exact mode runs the tail with one thread per row instead.
template <typename W>
__device__ __forceinline__ void anb_rate_coo_atomic(int nnz, const int* __restrict__ rows,
                                                    const int* __restrict__ cols,
                                                    const W* __restrict__ w,
                                                    const float* __restrict__ pre_r,
                                                    const int* __restrict__ post_rank,
                                                    float* __restrict__ sum) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += gridDim.x * blockDim.x) {
    const int row = rows[k];
    const int post = post_rank ? post_rank[row] : row;
    atomicAdd(&sum[post], pre_r[cols[k]] * anb_wf(w[k]));
  }
}

// ---- panelled sliced ELL (fast mode) ------------------------------------------------
// The pre-synaptic columns are cut into panels of at most `panel_width`
// neurons (16-bit column indices relative to the panel). Within a panel the
// rows are sorted by their number of synapses there and cut into slices of 32
// rows stored as steps of 32 elements, one per row: a header step naming the
// rows, then element k of every row at step k + 1. A CTA copies its panel's
// rates into shared memory with bulk (TMA) copies; each warp then streams a
// contiguous range of steps, one row per lane, loading the next chunk of U
// steps while it sums the current one, and adds its partial sum to the row's
// global sum where a slice (or its range) ends.

// Issue bulk copies of `bytes` (a multiple of 16, both addresses 16-byte
// aligned) from global memory into this CTA's shared memory, completing on
// the mbarrier `mbar` (phase 0). Called by one thread; the barrier must be
// published (CTA barrier) before other threads wait on it.
__device__ __forceinline__ void anb_bulk_issue(void* dst, const void* src, unsigned bytes,
                                               unsigned long long* mbar) {
  const unsigned mb = (unsigned)__cvta_generic_to_shared(mbar);
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("{ .reg .b64 st; mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1; }"
               ::"r"(mb), "r"(bytes) : "memory");
  const unsigned chunk = 32768u;
  for (unsigned off = 0; off < bytes; off += chunk) {
    const unsigned n = bytes - off < chunk ? bytes - off : chunk;
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(d + off), "l"(reinterpret_cast<const char*>(src) + off), "r"(n), "r"(mb)
        : "memory");
  }
}

// Wait for phase 0 of `mbar`, at most ANB_BULK_WAIT_TRIES polls; a timeout is
// reported in `err` (the copied data is then incomplete; the kernel still
// finishes).
#define ANB_BULK_WAIT_TRIES (1 << 22)
__device__ __forceinline__ void anb_bulk_wait(unsigned long long* mbar, int* err) {
  const unsigned mb = (unsigned)__cvta_generic_to_shared(mbar);
  unsigned done = 0;
  for (int it = 0; it < ANB_BULK_WAIT_TRIES && !done; ++it) {
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0; selp.u32 %0, 1, 0, p; }"
        : "=r"(done) : "r"(mb) : "memory");
  }
  if (!done) anb_report(err, ANB_DEVERR_BARRIER_TIMEOUT);
}

// Eight consecutive weights (aligned) widened to float.
__device__ __forceinline__ void anb_w8(const float* w, float* o) {
  const float4 a = anb_ls_f4(reinterpret_cast<const float4*>(w));
  const float4 b = anb_ls_f4(reinterpret_cast<const float4*>(w) + 1);
  o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w; o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
}
__device__ __forceinline__ void anb_w8(const anb_bf16* w, float* o) {
  const uint4 u = anb_ls_u4(reinterpret_cast<const uint4*>(w));
  const anb_u32 q[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    o[2 * i] = __uint_as_float(q[i] << 16);
    o[2 * i + 1] = __uint_as_float(q[i] & 0xffff0000u);
  }
}

// Sum index of a header entry (column c, weight slot read as wv): the entry
// stores v = index + 1 (0 for a padding lane) as column 0xF000 | (v >> 16)
// and the weight slot's bits v (32-bit weights) or v & 0xffff (bfloat16).
__device__ __forceinline__ int anb_pc_row(unsigned c, float wv, const float*) {
  return __float_as_int(wv) - 1;
}
__device__ __forceinline__ int anb_pc_row(unsigned c, float wv, const anb_bf16*) {
  return (int)(((c & 0xfffu) << 16) | (__float_as_uint(wv) >> 16)) - 1;
}

// cta_panel[blockIdx.x]: the CTA's panel; warp_tab[3 * (blockIdx.x * warps
// + warp) ...] = (first step, end step, header step of the slice holding the
// first step); col / w: 32 entries per step, columns from 0xF000 on marking
// header steps. Dynamic shared memory: panel_width floats.
// Weight of a pcsr entry as float (streaming load; the compiler folds the
// constant step offsets of a chunk into the load addresses).
__device__ __forceinline__ float anb_pc_w(const float* w) { return __ldcs(w); }
__device__ __forceinline__ float anb_pc_w(const anb_bf16* w) {
  return __uint_as_float((unsigned)__ldcs(reinterpret_cast<const unsigned short*>(w)) << 16);
}

template <typename W, int U>
__device__ __forceinline__ void anb_rate_pcsr(const int* __restrict__ cta_panel,
                                              const int* __restrict__ warp_tab,
                                              const unsigned short* __restrict__ col,
                                              const W* __restrict__ w,
                                              const float* __restrict__ x, int n_pre,
                                              int panel_width, float* __restrict__ sum, int* err) {
  extern __shared__ __align__(16) unsigned char anb_pc_smem[];
  __shared__ __align__(8) unsigned long long anb_pc_mbar;
  float* xs = reinterpret_cast<float*>(anb_pc_smem);
  const int p = cta_panel[blockIdx.x];
  const int c0 = p * panel_width;
  const int cw = min(panel_width, n_pre - c0);
  const int cw4 = cw & ~3;
  if (threadIdx.x == 0 && cw4 > 0) anb_bulk_issue(xs, x + c0, 4u * (unsigned)cw4, &anb_pc_mbar);
  for (int q = cw4 + threadIdx.x; q < cw; q += blockDim.x) xs[q] = x[c0 + q];
  const int lane = threadIdx.x & 31;
  const int* wt = warp_tab + 3 * (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
  const int sb = wt[0], se = wt[1], hd = wt[2];
  const unsigned short* __restrict__ cp = col + 32ll * sb + lane;
  const W* __restrict__ wp = w + 32ll * sb + lane;
  unsigned short ca[U], cb[U];
  float wa[U], wb[U];
  // the U steps from step j: all of them (full) or those before se; a step
  // past the range reads as a padding header (no row), which ends the lane's
  // current row there; the range test is warp-uniform
  auto load = [&](unsigned short (&c)[U], float (&wv)[U], const int j) {
    const unsigned short* cq = cp + 32 * (j - sb);
    const W* wq = wp + 32 * (j - sb);
    if (j + U <= se) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        c[u] = __ldcs(cq + 32 * u);
        wv[u] = anb_pc_w(wq + 32 * u);
      }
    } else {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const bool in = j + u < se;
        c[u] = in ? __ldcs(cq + 32 * u) : (unsigned short)0xf000u;
        wv[u] = in ? anb_pc_w(wq + 32 * u) : 0.f;
      }
    }
  };
  float acc = 0.f;
  int cur = -1;                                      // sum index of the lane's current row
  auto consume = [&](const unsigned short (&c)[U], const float (&wv)[U]) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (c[u] >= 0xf000u) {                         // header: the previous slice ends
        if (cur >= 0) atomicAdd(&sum[cur], acc);
        acc = 0.f;
        cur = anb_pc_row(c[u], wv[u], w);
      } else {
        acc = fmaf(xs[c[u]], wv[u], acc);
      }
    }
  };
  if (sb < se) {                                     // in flight during the panel copy
    load(ca, wa, sb);
    if (hd < sb) cur = anb_pc_row(anb_ls_h(col + 32ll * hd + lane), anb_w1(w + 32ll * hd + lane), w);
  }
  __syncthreads();                                   // mbarrier and tail rates published
  if (cw4 > 0) anb_bulk_wait(&anb_pc_mbar, err);
  for (int j = sb; j < se; j += 2 * U) {
    load(cb, wb, j + U);
    consume(ca, wa);
    load(ca, wa, j + 2 * U);
    consume(cb, wb);
  }
  if (cur >= 0) atomicAdd(&sum[cur], acc);
}

// ---- event-driven transmission -----------------------------------------------------

// Exact gather: thread per post row; g[post] += w[j] for every synapse whose
// pre neuron spiked, in row (ascending pre) order.
template <typename R, typename W>
__device__ __forceinline__ void anb_spike_gather(int n_rows, const int* __restrict__ row_ptr,
                                                 const int* __restrict__ col,
                                                 const W* __restrict__ w,
                                                 const anb_u32* __restrict__ spk,
                                                 const int* __restrict__ post_rank,
                                                 R* __restrict__ g) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n_rows;
       row += gridDim.x * blockDim.x) {
    const int beg = row_ptr[row], end = row_ptr[row + 1];
    const int post = post_rank ? post_rank[row] : row;
    R acc = g[post];
    bool any = false;
    for (int j = beg; j < end; ++j) {
      if (anb_bit(spk, col[j])) {
        acc += (R)w[j];
        any = true;
      }
    }
    if (any) g[post] = acc;
  }
}

// Exact gather, warp per post row: lanes test 32 synapses at a time; the
// spiking ones are added in ascending pre rank (set bits of the ballot in
// order), which is the reference's per-post order.
template <typename R, typename W>
__device__ __forceinline__ void anb_spike_gather_warp(int n_rows, const int* __restrict__ row_ptr,
                                                      const int* __restrict__ col,
                                                      const W* __restrict__ w,
                                                      const anb_u32* __restrict__ spk,
                                                      const int* __restrict__ post_rank,
                                                      R* __restrict__ g) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int row = warp; row < n_rows; row += nwarps) {
    const int beg = row_ptr[row], end = row_ptr[row + 1];
    const int post = post_rank ? post_rank[row] : row;
    R acc = g[post];
    bool any = false;
    for (int base = beg; base < end; base += 32) {
      const int j = base + lane;
      const bool sp = j < end && anb_bit(spk, col[j]);
      anb_u32 m = __ballot_sync(0xffffffffu, sp);
      any |= m != 0u;
      const R wj = sp ? (R)w[j] : R(0);
      while (m) {
        const int b = __ffs(m) - 1;
        m &= m - 1;
        acc += __shfl_sync(0xffffffffu, wj, b);
      }
    }
    if (any && lane == 0) g[post] = acc;
  }
}

// Spike transmission with one delay per synapse (steps, 1..dmax): warp per
// post row; a spike emitted at step s reaches the synapses of delay t - s at
// step t. `ring` holds one spike bitmap of `words` words per step, `slots`
// steps. ORDERED adds the contributions one at a time in the reference's
// order: emission step ascending, then pre rank ascending (the push order of
// its ring of delayed spikes, ANNarchy/generator/Projection/SingleThread/
// LIL.py:915-969): a first pass over the row collects the delays that
// deliver a spike this step (a bit mask), then one pass per such delay, the
// largest first. Without ORDERED one pass adds them in pre-rank order.
template <typename R, typename W, bool ORDERED>
__device__ __forceinline__ void anb_spike_gather_delayed(int n_rows, const int* __restrict__ row_ptr,
                                                         const int* __restrict__ col,
                                                         const W* __restrict__ w,
                                                         const int* __restrict__ dly,
                                                         const anb_u32* __restrict__ ring, int words,
                                                         int slots, long long t,
                                                         const int* __restrict__ post_rank,
                                                         R* __restrict__ g) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int row = warp; row < n_rows; row += nwarps) {
    const int beg = row_ptr[row], end = row_ptr[row + 1];
    const int post = post_rank ? post_rank[row] : row;
    // delays (bit d) that deliver a spike to this row at step t
    unsigned long long dmask = 0ull;
    R acc = g[post];
    for (int base = beg; base < end; base += 32) {
      const int j = base + lane;
      bool sp = false;
      int d = 0;
      if (j < end) {
        d = dly[j];
        sp = anb_bit(ring + (size_t)anb_ring_slot(t - d, slots) * words, col[j]);
      }
      if (ORDERED) {
        unsigned long long m = sp ? (1ull << d) : 0ull;
        for (int o = 16; o > 0; o >>= 1) m |= __shfl_xor_sync(0xffffffffu, m, o);
        dmask |= m;
      } else {
        anb_u32 m = __ballot_sync(0xffffffffu, sp);
        dmask |= m;
        const R wj = sp ? (R)w[j] : R(0);
        while (m) {
          const int b = __ffs(m) - 1;
          m &= m - 1;
          acc += __shfl_sync(0xffffffffu, wj, b);
        }
      }
    }
    if (ORDERED) {
      for (unsigned long long rest = dmask; rest; ) {
        const int d = 63 - __clzll(rest);              // largest delay first: oldest spikes
        rest &= ~(1ull << d);
        const anb_u32* spk = ring + (size_t)anb_ring_slot(t - d, slots) * words;
        for (int base = beg; base < end; base += 32) {
          const int j = base + lane;
          const bool sp = j < end && dly[j] == d && anb_bit(spk, col[j]);
          anb_u32 m = __ballot_sync(0xffffffffu, sp);
          const R wj = sp ? (R)w[j] : R(0);
          while (m) {
            const int b = __ffs(m) - 1;
            m &= m - 1;
            acc += __shfl_sync(0xffffffffu, wj, b);
          }
        }
      }
    }
    if (dmask != 0ull && lane == 0) g[post] = acc;
  }
}

// Fast scatter: a warp per 32-neuron bitmap word of the pre population
// (words [w0, w1)); for every set bit the warp walks that neuron's outgoing
// synapses (pre-major: col_ptr / post_idx / w_pre) and adds w to g[post]
// with atomics. Warp-uniform control flow; lanes stride the fan-out.
template <typename R, typename W>
__device__ __forceinline__ void anb_spike_scatter(int w0, int w1, const anb_u32* __restrict__ spk,
                                                  const int* __restrict__ col_ptr,
                                                  const int* __restrict__ post_idx,
                                                  const W* __restrict__ w_pre,
                                                  R* __restrict__ g) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int word = w0 + warp; word < w1; word += nwarps) {
    anb_u32 m = spk[word];
    while (m) {
      const int b = __ffs(m) - 1;
      m &= m - 1;
      const int pre = (word << 5) + b;
      const int beg = col_ptr[pre], end = col_ptr[pre + 1];
      for (int k = beg + lane; k < end; k += 32) atomicAdd(&g[post_idx[k]], (R)anb_wf(w_pre[k]));
    }
  }
}

// ---- thread-block clusters (distributed shared memory) ----------------------------------
// The cluster engine splits a network's neurons over the CTAs of one
// cluster; spikes are delivered into the owning CTA's shared memory with
// DSMEM reductions and the CTAs meet at one hardware cluster barrier per
// step (no spin loop).

__device__ __forceinline__ unsigned anb_cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

__device__ __forceinline__ unsigned anb_smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

// Address of the same shared-memory offset in CTA `rank` of the cluster.
__device__ __forceinline__ unsigned anb_cluster_map(unsigned addr, unsigned rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}

__device__ __forceinline__ void anb_cluster_red_add(unsigned addr, float v) {
  asm volatile("red.relaxed.cluster.shared::cluster.add.f32 [%0], %1;" ::"r"(addr), "f"(v)
               : "memory");
}

__device__ __forceinline__ void anb_cluster_st_u32(unsigned addr, anb_u32 v) {
  asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}

__device__ __forceinline__ void anb_cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::
                   : "memory");
}

// Fast scatter from a spike list: work item = (spike, 32-synapse chunk of its
// fan-out), so a warp does one pass per item whatever the fan-out; spikes
// outside [lo, hi) (not pre neurons of this projection) are skipped.
template <typename R, typename W>
__device__ __forceinline__ void anb_spike_scatter_list(int lo, int hi, const int* __restrict__ list,
                                                       int count, int chunks,
                                                       const int* __restrict__ col_ptr,
                                                       const int* __restrict__ post_idx,
                                                       const W* __restrict__ w_pre,
                                                       R* __restrict__ g) {
  const int lane = threadIdx.x & 31;
  const long long items = (long long)count * chunks;
  for (long long it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < items;
       it += (gridDim.x * blockDim.x) >> 5) {
    const int pre = list[it / chunks];
    if (pre < lo || pre >= hi) continue;
    const int c = (int)(it % chunks);
    const int end = col_ptr[pre + 1];
    for (int q = col_ptr[pre] + c * 32 + lane; q < end; q += 32 * chunks)
      atomicAdd(&g[post_idx[q]], (R)anb_wf(w_pre[q]));
  }
}

// ---- grid-wide barrier of a cooperative persistent launch ----------------------------
// bar[0] counts the CTAs that arrived, bar[1] is the generation. Every CTA
// reads the generation before arriving; the last to arrive resets the count
// and advances the generation, the others wait (bounded by a cycle budget of
// about one second) until it changes. Returns false when this or any other
// CTA gave up (err[0] holds ANB_DEVERR_BARRIER_TIMEOUT): the caller leaves its
// loop. Other device errors (a full monitor ring) do not stop the run.
#define ANB_GRID_WAIT_CYCLES (2000000000ll)
__device__ __forceinline__ bool anb_grid_sync(unsigned* bar, int* err) {
  __shared__ int anb_gs_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = bar + 1;
    const unsigned g = *gen;
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u);
    int ok = 1;
    if (arrived == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const long long c0 = clock64();
      while (*gen == g) {
        if (clock64() - c0 > ANB_GRID_WAIT_CYCLES ||
            *(volatile int*)err == ANB_DEVERR_BARRIER_TIMEOUT) {
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
      if (!ok) atomicExch(err, ANB_DEVERR_BARRIER_TIMEOUT);
    }
    __threadfence();
    anb_gs_ok = ok && *(volatile int*)err != ANB_DEVERR_BARRIER_TIMEOUT;
  }
  __syncthreads();
  return anb_gs_ok != 0;
}

// ---- monitors ---------------------------------------------------------------------------

// Copy n values (converted to double) into slot `slot` of a ring of `cap` slots.
template <typename T>
__device__ __forceinline__ void anb_record(const T* __restrict__ src, const int* __restrict__ ranks,
                                           int n, double* __restrict__ buf, long long slot) {
  double* dst = buf + slot * (long long)n;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    dst[k] = (double)src[ranks ? ranks[k] : k];
}


// Exclusive prefix sum of x over the CTA (blockDim.x a multiple of 32, at
// most 1024). `warp_sums` is 32 ints of shared memory; two CTA barriers.
__device__ __forceinline__ int anb_block_exclusive_scan(int x, int* warp_sums, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int s = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += v;
    }
    if (lane < nw) warp_sums[lane] = s;
  }
  __syncthreads();
  *total = warp_sums[nw - 1];
  return (warp ? warp_sums[warp - 1] : 0) + incl - x;
}
