// Device-side connectivity construction, included at the end of runtime.cu
// (it creates named arrays of a network).
//
// The reference builds every projection on the host as a list of lists
// (ANNarchy/cython_ext/Connector.pyx:93-420) and uploads it; for 1e9
// synapses that takes longer than the simulation. Here a fixed in-degree
// projection is generated where it lives.
//
// Sampling: the pre range [pre_lo, pre_hi) is cut into `number` equal strata
// and one pre neuron is drawn in every stratum, so each row holds `number`
// distinct pre ranks in ascending order (the reference draws a uniformly
// random subset; the in-degree is the same). Random numbers come from a
// counter-based hash of (seed, row, slot, stream) with the SplitMix64
// finaliser (Steele, Lea and Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014).

namespace {

__device__ __forceinline__ unsigned long long anb_mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ double anb_u01(unsigned long long seed, long long row, int slot,
                                          int stream) {
  unsigned long long h = anb_mix64(seed ^ anb_mix64((unsigned long long)row * 0x100000001B3ull +
                                                    (unsigned long long)slot * 4 + stream));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);   // 53 random bits in [0, 1)
}

template <typename W>
__device__ __forceinline__ W anb_from_double(double v) {
  return (W)v;
}
template <>
__device__ __forceinline__ unsigned short anb_from_double<unsigned short>(double v) {
  unsigned int u = __float_as_uint((float)v);
  u += 0x7FFFu + ((u >> 16) & 1u);                          // round to nearest even
  return (unsigned short)(u >> 16);
}

template <typename W>
__global__ void anb_fixed_number_pre_kernel(int n_post, int post_base, long long row_offset,
                                            int pre_lo, int pre_hi,
                                            int number, unsigned long long seed, int wkind,
                                            double a, double b, int exclude_self,
                                            int* __restrict__ post_rank, int* __restrict__ row_ptr,
                                            int* __restrict__ col, W* __restrict__ w) {
  const long long total = (long long)n_post * number;
  const double width = (double)(pre_hi - pre_lo) / number;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long row = e / number;
    const long long grow = row_offset + row;                  // row of the whole projection
    const int k = (int)(e - row * number);
    const int s0 = pre_lo + (int)floor(k * width);
    int s1 = pre_lo + (int)floor((k + 1) * width);
    if (s1 <= s0) s1 = s0 + 1;
    int pre = s0 + (int)(anb_u01(seed, grow, k, 0) * (s1 - s0));
    if (pre >= s1) pre = s1 - 1;
    const int post = post_base + (int)row;
    if (exclude_self && pre == post) pre = (pre + 1 < s1) ? pre + 1 : (pre - 1 >= s0 ? pre - 1 : pre);
    col[e] = pre;
    double v = a;
    if (wkind == 1) {
      v = a + (b - a) * anb_u01(seed, grow, k, 1);
    } else if (wkind == 2) {                                // Box-Muller
      const double u1 = 1.0 - anb_u01(seed, grow, k, 1), u2 = anb_u01(seed, grow, k, 2);
      v = a + b * sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
    }
    w[e] = anb_from_double<W>(v);
    if (k == 0) {
      row_ptr[row] = (int)e;
      post_rank[row] = post;
    }
    if (e == total - 1) row_ptr[n_post] = (int)total;
  }
}

__global__ void anb_count_cols(const int* __restrict__ col, long long nnz, int* __restrict__ cnt) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < nnz;
       j += (long long)gridDim.x * blockDim.x)
    atomicAdd(&cnt[col[j] + 1], 1);
}

// In-place inclusive scan of n ints with one CTA (cnt[0] = 0 gives the
// exclusive column pointers).
__global__ void anb_scan_single_cta(int* __restrict__ v, int n) {
  __shared__ int part[1024];
  const int per = (n + blockDim.x - 1) / blockDim.x;
  const int lo = threadIdx.x * per, hi = min(n, lo + per);
  int s = 0;
  for (int i = lo; i < hi; ++i) s += v[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < (int)blockDim.x; o <<= 1) {
    const int y = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += y;
    __syncthreads();
  }
  int run = threadIdx.x ? part[threadIdx.x - 1] : 0;
  for (int i = lo; i < hi; ++i) {
    run += v[i];
    v[i] = run;
  }
}

template <typename W>
__global__ void anb_scatter_cols(int n_rows, const int* __restrict__ row_ptr,
                                 const int* __restrict__ col, const int* __restrict__ post_rank,
                                 const W* __restrict__ w, int* __restrict__ cursor,
                                 int* __restrict__ post_idx, int* __restrict__ inv_idx,
                                 W* __restrict__ w_pre) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n_rows;
       row += gridDim.x * blockDim.x) {
    const int post = post_rank[row];
    for (int j = row_ptr[row]; j < row_ptr[row + 1]; ++j) {
      const int pos = atomicAdd(&cursor[col[j]], 1);
      post_idx[pos] = post;
      inv_idx[pos] = j;
      if (w_pre) w_pre[pos] = w[j];
    }
  }
}

__global__ void anb_fill_kernel(unsigned char* __restrict__ dst, size_t bytes,
                                const unsigned long long pattern, const unsigned long long pattern_hi,
                                int pattern_bytes) {
  const size_t n = bytes / pattern_bytes;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    if (pattern_bytes == 16) reinterpret_cast<ulonglong2*>(dst)[i] = make_ulonglong2(pattern, pattern_hi);
    else if (pattern_bytes == 8) reinterpret_cast<unsigned long long*>(dst)[i] = pattern;
    else if (pattern_bytes == 4) reinterpret_cast<unsigned int*>(dst)[i] = (unsigned int)pattern;
    else if (pattern_bytes == 2) reinterpret_cast<unsigned short*>(dst)[i] = (unsigned short)pattern;
    else dst[i] = (unsigned char)pattern;
  }
}

// dst[i * dst_stride + dst_off] = src[i * src_stride + src_off] for 4-byte
// elements (strides and offsets in 4-byte words).
__global__ void anb_copy_strided_kernel(unsigned* __restrict__ dst, long long dst_stride, long long dst_off,
                                        const unsigned* __restrict__ src, long long src_stride,
                                        long long src_off, long long count) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x)
    dst[i * dst_stride + dst_off] = src[i * src_stride + src_off];
}

unsigned grid_of(long long n) {
  long long g = (n + 255) / 256;
  return (unsigned)(g < 1 ? 1 : (g > 148 * 32 ? 148 * 32 : g));
}

}  // namespace

extern "C" {

int anb_array_fill(anb_net* net, const char* name, const void* value, size_t value_bytes) {
  if (!net || !value) return fail(ANB_ERR_ARG, "NULL argument");
  if (value_bytes != 1 && value_bytes != 2 && value_bytes != 4 && value_bytes != 8 && value_bytes != 16)
    return fail(ANB_ERR_ARG, "fill value must be 1, 2, 4, 8 or 16 bytes");
  Array* a = find(net, name);
  if (!a) return fail(ANB_ERR_ARG, std::string("unknown array ") + (name ? name : "(null)"));
  if (a->bytes % value_bytes) return fail(ANB_ERR_ARG, "array size is not a multiple of the value");
  int rc = ensure_device(net);
  if (rc) return rc;
  unsigned long long pattern[2] = {0, 0};
  std::memcpy(pattern, value, value_bytes);
  if (a->bytes) {
    anb_fill_kernel<<<grid_of((long long)(a->bytes / value_bytes)), 256, 0, net->stream>>>(
        (unsigned char*)a->ptr, a->bytes, pattern[0], pattern[1], (int)value_bytes);
    ANB_CUDA(cudaGetLastError());
  }
  ANB_CUDA(cudaStreamSynchronize(net->stream));
  return ANB_OK;
}

int anb_array_copy_strided(anb_net* net, const char* dst, size_t dst_offset, size_t dst_stride,
                           const char* src, size_t src_offset, size_t src_stride, size_t count) {
  if (!net || !dst || !src) return fail(ANB_ERR_ARG, "NULL argument");
  Array* d = find(net, dst);
  Array* a = find(net, src);
  if (!d || !a) return fail(ANB_ERR_ARG, "unknown array");
  if ((dst_offset | dst_stride | src_offset | src_stride) % 4 || dst_stride == 0 || src_stride == 0)
    return fail(ANB_ERR_ARG, "offsets and strides must be multiples of 4 bytes");
  if (count == 0) return ANB_OK;
  if (dst_offset + (count - 1) * dst_stride + 4 > d->bytes ||
      src_offset + (count - 1) * src_stride + 4 > a->bytes)
    return fail(ANB_ERR_ARG, "strided copy outside an array");
  int rc = ensure_device(net);
  if (rc) return rc;
  anb_copy_strided_kernel<<<grid_of((long long)count), 256, 0, net->stream>>>(
      (unsigned*)d->ptr, (long long)(dst_stride / 4), (long long)(dst_offset / 4), (const unsigned*)a->ptr,
      (long long)(src_stride / 4), (long long)(src_offset / 4), (long long)count);
  ANB_CUDA(cudaGetLastError());
  ANB_CUDA(cudaStreamSynchronize(net->stream));
  return ANB_OK;
}

int anb_connect_fixed_number_pre(anb_net* net, const char* prefix, int n_post, int post_base,
                                 int pre_lo, int pre_hi, int number, uint64_t seed,
                                 int weight_kind, double a, double b, int weight_bytes,
                                 int exclude_self) {
  return anb_connect_fixed_number_pre_rows(net, prefix, n_post, post_base, 0, pre_lo, pre_hi, number,
                                           seed, weight_kind, a, b, weight_bytes, exclude_self);
}

int anb_connect_fixed_number_pre_rows(anb_net* net, const char* prefix, int n_post, int post_base,
                                      long long row_offset, int pre_lo, int pre_hi, int number,
                                      uint64_t seed, int weight_kind, double a, double b,
                                      int weight_bytes, int exclude_self) {
  if (!net || !prefix || row_offset < 0) return fail(ANB_ERR_ARG, "NULL argument or negative row offset");
  if (n_post <= 0 || number <= 0 || pre_hi - pre_lo < number || weight_kind < 0 || weight_kind > 2)
    return fail(ANB_ERR_ARG, "bad fixed_number_pre arguments");
  const long long nnz = (long long)n_post * number;
  if (nnz >= (1ll << 31)) return fail(ANB_ERR_ARG, "more than 2^31-1 synapses in one projection");
  if (weight_bytes != 8 && weight_bytes != 4 && weight_bytes != 2)
    return fail(ANB_ERR_ARG, "weight_bytes must be 8, 4 or 2");
  int rc = ensure_device(net);
  if (rc) return rc;
  const std::string p(prefix);
  if ((rc = create_array(net, p + "__post_rank", (size_t)n_post * 4))) return rc;
  if ((rc = create_array(net, p + "__row_ptr", (size_t)(n_post + 1) * 4))) return rc;
  if ((rc = create_array(net, p + "__col", (size_t)nnz * 4))) return rc;
  if ((rc = create_array(net, p + "__w", (size_t)nnz * weight_bytes))) return rc;
  int* pr = (int*)find(net, (p + "__post_rank").c_str())->ptr;
  int* rp = (int*)find(net, (p + "__row_ptr").c_str())->ptr;
  int* cl = (int*)find(net, (p + "__col").c_str())->ptr;
  void* w = find(net, (p + "__w").c_str())->ptr;
  const unsigned g = grid_of(nnz);
  if (weight_bytes == 8)
    anb_fixed_number_pre_kernel<double><<<g, 256, 0, net->stream>>>(
        n_post, post_base, row_offset, pre_lo, pre_hi, number, seed, weight_kind, a, b, exclude_self, pr, rp, cl,
        (double*)w);
  else if (weight_bytes == 4)
    anb_fixed_number_pre_kernel<float><<<g, 256, 0, net->stream>>>(
        n_post, post_base, row_offset, pre_lo, pre_hi, number, seed, weight_kind, a, b, exclude_self, pr, rp, cl,
        (float*)w);
  else
    anb_fixed_number_pre_kernel<unsigned short><<<g, 256, 0, net->stream>>>(
        n_post, post_base, row_offset, pre_lo, pre_hi, number, seed, weight_kind, a, b, exclude_self, pr, rp, cl,
        (unsigned short*)w);
  ANB_CUDA(cudaGetLastError());
  ANB_CUDA(cudaStreamSynchronize(net->stream));
  return ANB_OK;
}

int anb_csr_to_csc(anb_net* net, const char* prefix, int n_pre, int with_weights) {
  if (!net || !prefix || n_pre <= 0) return fail(ANB_ERR_ARG, "bad argument");
  int rc = ensure_device(net);
  if (rc) return rc;
  const std::string p(prefix);
  Array* rp = find(net, (p + "__row_ptr").c_str());
  Array* cl = find(net, (p + "__col").c_str());
  Array* pr = find(net, (p + "__post_rank").c_str());
  Array* w = find(net, (p + "__w").c_str());
  if (!rp || !cl || !pr || !w) return fail(ANB_ERR_ARG, "CSR arrays of " + p + " missing");
  const int n_rows = (int)(pr->bytes / 4);
  const long long nnz = (long long)(cl->bytes / 4);
  const size_t wb = nnz ? w->bytes / (size_t)nnz : 4;
  if ((rc = create_array(net, p + "__col_ptr", (size_t)(n_pre + 1) * 4))) return rc;
  if ((rc = create_array(net, p + "__post_idx", (size_t)nnz * 4))) return rc;
  if ((rc = create_array(net, p + "__inv_idx", (size_t)nnz * 4))) return rc;
  if (with_weights && (rc = create_array(net, p + "__w_pre", (size_t)nnz * wb))) return rc;
  rp = find(net, (p + "__row_ptr").c_str());
  cl = find(net, (p + "__col").c_str());
  pr = find(net, (p + "__post_rank").c_str());
  w = find(net, (p + "__w").c_str());
  int* cp = (int*)find(net, (p + "__col_ptr").c_str())->ptr;
  int* pi = (int*)find(net, (p + "__post_idx").c_str())->ptr;
  int* ii = (int*)find(net, (p + "__inv_idx").c_str())->ptr;
  void* wp = with_weights ? find(net, (p + "__w_pre").c_str())->ptr : nullptr;
  anb_count_cols<<<grid_of(nnz), 256, 0, net->stream>>>((const int*)cl->ptr, nnz, cp);
  anb_scan_single_cta<<<1, 1024, 0, net->stream>>>(cp, n_pre + 1);
  int* cursor = nullptr;
  ANB_CUDA(cudaMalloc(&cursor, (size_t)(n_pre + 1) * 4));
  cudaMemcpyAsync(cursor, cp, (size_t)(n_pre + 1) * 4, cudaMemcpyDeviceToDevice, net->stream);
  if (wb == 8)
    anb_scatter_cols<double><<<grid_of(n_rows), 256, 0, net->stream>>>(
        n_rows, (const int*)rp->ptr, (const int*)cl->ptr, (const int*)pr->ptr, (const double*)w->ptr,
        cursor, pi, ii, (double*)wp);
  else if (wb == 4)
    anb_scatter_cols<float><<<grid_of(n_rows), 256, 0, net->stream>>>(
        n_rows, (const int*)rp->ptr, (const int*)cl->ptr, (const int*)pr->ptr, (const float*)w->ptr,
        cursor, pi, ii, (float*)wp);
  else
    anb_scatter_cols<unsigned short><<<grid_of(n_rows), 256, 0, net->stream>>>(
        n_rows, (const int*)rp->ptr, (const int*)cl->ptr, (const int*)pr->ptr,
        (const unsigned short*)w->ptr, cursor, pi, ii, (unsigned short*)wp);
  cudaError_t e = cudaGetLastError();
  cudaStreamSynchronize(net->stream);
  cudaFree(cursor);
  if (e != cudaSuccess) return fail(ANB_ERR_CUDA, std::string("csr_to_csc: ") + cudaGetErrorString(e));
  return ANB_OK;
}

}  // extern "C"
