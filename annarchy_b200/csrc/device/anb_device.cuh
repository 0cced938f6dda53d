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
#define ANB_DEVERR_BARRIER_TIMEOUT 1
#define ANB_DEVERR_INDEX 2
#define ANB_DEVERR_MONITOR_OVERFLOW 3

// ---- built-in functions of the equation language --------------------------
// (names as emitted by the reference parser: ANNarchy/parser/ParserTemplate.py)
template <typename T> __device__ __forceinline__ T positive(T x) { return x > T(0) ? x : T(0); }
template <typename T> __device__ __forceinline__ T negative(T x) { return x < T(0) ? x : T(0); }
__device__ __forceinline__ double modulo(double a, double b) { return fmod(a, b); }
__device__ __forceinline__ int modulo(int a, int b) { return a % b; }
__device__ __forceinline__ double power(double a, double b) { return pow(a, b); }
__device__ __forceinline__ float power(float a, float b) { return powf(a, b); }
#define clip(x, a, b) ((x) < (a) ? (a) : ((x) > (b) ? (b) : (x)))

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
    for (int k = 0; k < len; ++k) {
      const int c = cols[(size_t)k * n_rows + row];
      if (!rl && c < 0) break;
      s += pre_r[c] * (R)anb_wf(w[(size_t)k * n_rows + row]);
    }
    const int post = post_rank ? post_rank[row] : row;
    sum[post] += s;
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
    for (int k = 0; k < len; ++k) {
      const int slot = base + k * C + lane;
      s += pre_r[cols[slot]] * (R)anb_wf(w[slot]);
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

// ---- monitors ---------------------------------------------------------------------------

// Copy n values (converted to double) into slot `slot` of a ring of `cap` slots.
template <typename T>
__device__ __forceinline__ void anb_record(const T* __restrict__ src, const int* __restrict__ ranks,
                                           int n, double* __restrict__ buf, long long slot) {
  double* dst = buf + slot * (long long)n;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    dst[k] = (double)src[ranks ? ranks[k] : k];
}
