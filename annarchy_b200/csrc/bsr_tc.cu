// Batched weighted sums over dense 64 x 64 blocks on the 5th-generation
// tensor cores (tcgen05): Y[b][post] += sum over the nonzero blocks of a
// block-sparse (BSR) matrix W (post x pre, bfloat16) times the rates X[b][pre]
// of `batch` instances (bfloat16 operands, float accumulation).
//
// The reference's BSR container and its per-instance weighted sum
// (ANNarchy/include/BSRMatrix.hpp:41, ANNarchy/generator/Projection/CUDA/BSR.py:296)
// compute one vector per launch; with many instances sharing the weights
// (parameter sweeps of a rate-coded network) every block becomes a 64 x 64 x B
// matrix product, which belongs on the tensor cores.
//
// Kernel bsr_spmm_tc_kernel: one CTA (one warpgroup, 128 threads) per block row.
// One thread streams the row's blocks through a STAGES-deep ring of shared-
// memory stages with bulk copies (cp.async.bulk, completing on an mbarrier
// per stage; no multicast); another thread issues per block four tcgen05.mma of
// M=64, N=batch, K=16 (kind::f16, bf16 x bf16 -> f32) that accumulate in
// tensor memory; tcgen05.commit releases each stage when its products are
// done. The four warps then read the accumulator with tcgen05.ld (warp w owns
// rows 16w..16w+15 of the 64-row tile: lanes 0-15 of TMEM sub-partition w)
// and add it into Y. Every mbarrier wait is bounded: a timeout sets the error
// word, the CTA waits (bounded) for its outstanding copies and products, frees
// its tensor memory and returns.
//
// Operand layout in memory is the tcgen05 canonical K-major layout without
// swizzle: 8 x 8 "core matrices" of 16-byte rows, core (i, j) of a tile at
// byte (8 i + j) * 128 (i: group of 8 rows, j: group of 8 along K), so one
// bulk copy of a tile lands it ready for the matrix descriptors (leading-
// dimension offset 128 B between K cores, stride offset 1024 B between row
// groups).
#include <cstdint>
#include <cuda_runtime.h>

#include "device/anb_device.cuh"

namespace {

constexpr int kTile = 64;                 // block rows / columns
constexpr int kStages = 4;
constexpr unsigned kTileBytes = kTile * kTile * 2;   // 8 KB of bf16
constexpr int kWaitTries = 1 << 22;
constexpr int kColCache = 512;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("{ .reg .b64 st; mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1; }"
               ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Bounded wait for the phase of parity `parity`; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  const unsigned b = smem_u32(bar);
  unsigned done = 0;
  for (int it = 0; it < kWaitTries && !done; ++it) {
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done) : "r"(b), "r"(parity) : "memory");
  }
  return done != 0;
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

// Shared-memory matrix descriptor, K-major without swizzle: start address,
// leading-dimension byte offset (between the two K cores of one MMA), stride
// byte offset (between groups of 8 rows), version 1 (sm_100), layout type 0.
__device__ __forceinline__ uint64_t smem_desc(unsigned addr, unsigned lbo, unsigned sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: f32 accumulator, bf16 A and B, both K-major, dense.
__host__ __device__ constexpr uint32_t instr_desc(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                         uint32_t accumulate) {
  const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate),
        "r"(mask0), "r"(mask1), "r"(mask2), "r"(mask3));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__global__ void __launch_bounds__(128, 1)
bsr_spmm_tc_kernel(const int* __restrict__ brow_ptr, const int* __restrict__ bcol,
                const uint16_t* __restrict__ a_tiles, const uint16_t* __restrict__ x_tiles,
                int batch, float* __restrict__ y, int n_post, int tmem_cols, int* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t full[kStages], empty[kStages], done;
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag, issued_n, consumed_n;
  __shared__ int bcol_s[kColCache];        // the row's block columns (first kColCache)
  const unsigned x_bytes = (unsigned)batch * kTile * 2;
  const unsigned stage_bytes = kTileBytes + x_bytes;
  const int br = blockIdx.x;
  const int beg = brow_ptr[br], nblk = brow_ptr[br + 1] - beg;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(&tmem_base)), "r"(tmem_cols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
    issued_n = 0;
    consumed_n = 0;
  }
  for (int q = threadIdx.x; q < nblk && q < kColCache; q += blockDim.x) bcol_s[q] = bcol[beg + q];
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t taddr = tmem_base;

  // warp 0 lane 0 streams the blocks into the stage ring, warp 1 lane 0
  // issues the products as stages fill: neither waits on the other's latency
  if (nblk > 0 && threadIdx.x == 0) {
    int k = 0;
    for (; k < nblk; ++k) {
      const int s = k % kStages, u = k / kStages;
      if (u > 0 && !mbar_wait(&empty[s], (u - 1) & 1)) {
        anb_report(err, ANB_DEVERR_BARRIER_TIMEOUT);
        abort_flag = 1;
        break;
      }
      unsigned char* st = smem + s * stage_bytes;
      mbar_expect_tx(&full[s], stage_bytes);
      bulk_load(st, a_tiles + (size_t)(beg + k) * (kTile * kTile), kTileBytes, &full[s]);
      const int bc = k < kColCache ? bcol_s[k] : bcol[beg + k];
      bulk_load(st + kTileBytes, x_tiles + (size_t)bc * batch * kTile, x_bytes, &full[s]);
    }
    issued_n = k;
  } else if (nblk > 0 && threadIdx.x == 32) {
    const uint32_t idesc = instr_desc(kTile, batch);
    int k = 0;
    for (; k < nblk; ++k) {
      const int s = k % kStages, u = k / kStages;
      if (!mbar_wait(&full[s], u & 1)) {
        anb_report(err, ANB_DEVERR_BARRIER_TIMEOUT);
        abort_flag = 1;
        break;
      }
      const unsigned a0 = smem_u32(smem + s * stage_bytes);
      const unsigned b0 = a0 + kTileBytes;
#pragma unroll
      for (int q = 0; q < kTile / 16; ++q) {
        umma_f16(taddr, smem_desc(a0 + q * 256, 128, 1024), smem_desc(b0 + q * 256, 128, 1024),
                 idesc, (k > 0 || q > 0) ? 1u : 0u);
      }
      umma_commit(&empty[s]);
    }
    consumed_n = k;
    umma_commit(&done);                       // after every issued product
  }
  __syncthreads();
  if (abort_flag && threadIdx.x == 0) {
    // copies issued but never consumed: wait for them (bounded) before leaving
    for (int k = consumed_n; k < issued_n; ++k) mbar_wait(&full[k % kStages], (k / kStages) & 1);
  }
  __syncthreads();
  if (nblk > 0) {
    const bool ok = mbar_wait(&done, 0);
    if (!ok) anb_report(err, ANB_DEVERR_BARRIER_TIMEOUT);
    // uniform over the CTA: tcgen05.ld is executed by whole warps
    const int all_ok = __syncthreads_and(ok && !abort_flag ? 1 : 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (all_ok) {
      // warp w reads TMEM lanes 32w..32w+31; lanes 0-15 hold rows 16w..16w+15
      const int row = br * kTile + 16 * warp + lane;
      const bool mine = lane < 16 && row < n_post;
      for (int c0 = 0; c0 < batch; c0 += 16) {
        // the 16 loads of Y go out together (written before any store, so
        // they need not wait for one another) and overlap the tensor-memory read
        float old[16];
        uint32_t r[16];
        if (mine) {
#pragma unroll
          for (int j = 0; j < 16; ++j) old[j] = y[(size_t)(c0 + j) * n_post + row];
        }
        tmem_ld16(taddr + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, r);
        if (mine) {
#pragma unroll
          for (int j = 0; j < 16; ++j) y[(size_t)(c0 + j) * n_post + row] = old[j] + __uint_as_float(r[j]);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(tmem_cols)
                 : "memory");
  }
}

// The same products on the CUDA cores (the baseline the tensor-core kernel is
// measured against): one CTA of 256 threads per block row; thread t owns row
// t % 64 and PER = batch / 4 batch columns (in registers); tiles staged in
// shared memory as float.
template <int PER>
__global__ void __launch_bounds__(256)
bsr_spmm_simt_kernel(const int* __restrict__ brow_ptr, const int* __restrict__ bcol,
                     const uint16_t* __restrict__ a_tiles, const uint16_t* __restrict__ x_tiles,
                     float* __restrict__ y, int n_post) {
  constexpr int batch = 4 * PER;
  extern __shared__ __align__(1024) unsigned char smem[];
  float* as = reinterpret_cast<float*>(smem);                 // 64 x 64, row-major
  float* xs = as + kTile * kTile;                              // 64 x batch (k-major rows)
  const int br = blockIdx.x;
  const int beg = brow_ptr[br], end = brow_ptr[br + 1];
  const int r = threadIdx.x % kTile, part = threadIdx.x / kTile;
  float acc[PER];
#pragma unroll
  for (int j = 0; j < PER; ++j) acc[j] = 0.f;
  for (int blk = beg; blk < end; ++blk) {
    const uint16_t* at = a_tiles + (size_t)blk * kTile * kTile;
    const uint16_t* xt = x_tiles + (size_t)bcol[blk] * batch * kTile;
    __syncthreads();
    for (int e = threadIdx.x; e < kTile * kTile; e += blockDim.x) {
      // canonical layout -> row-major
      const int core = e >> 6, in = e & 63;
      const int row = (core >> 3) * 8 + (in >> 3), col = (core & 7) * 8 + (in & 7);
      as[row * kTile + col] = anb_bf16_to_f32(at[e]);
    }
    for (int e = threadIdx.x; e < batch * kTile; e += blockDim.x) {
      const int core = e >> 6, in = e & 63;
      const int b = (core >> 3) * 8 + (in >> 3), k = (core & 7) * 8 + (in & 7);
      xs[k * batch + b] = anb_bf16_to_f32(xt[e]);
    }
    __syncthreads();
    for (int k = 0; k < kTile; ++k) {
      const float a = as[r * kTile + k];
      const float* xk = xs + k * batch + part * PER;
#pragma unroll
      for (int j = 0; j < PER; ++j) acc[j] += a * xk[j];
    }
  }
  const int row = br * kTile + r;
  if (row < n_post && end > beg) {
#pragma unroll
    for (int j = 0; j < PER; ++j) y[(size_t)(part * PER + j) * n_post + row] += acc[j];
  }
}

// fp32 X[b][pre] -> bf16 tiles in the canonical layout (zero past n_pre).
// One thread per (instance, 8 consecutive neurons): a coalesced 32-byte read
// of X, one 16-byte row of a core matrix written.
__device__ __forceinline__ uint32_t bf16_pair(float lo, float hi) {
  const uint32_t a = __float_as_uint(lo), b = __float_as_uint(hi);
  const uint32_t ra = (a + 0x7FFFu + ((a >> 16) & 1u)) >> 16;   // round to nearest even
  const uint32_t rb = (b + 0x7FFFu + ((b >> 16) & 1u)) >> 16;
  return ra | (rb << 16);
}

__global__ void bsr_pack_x_kernel(const float* __restrict__ x, int batch, int n_pre, int n_bcols,
                                  uint16_t* __restrict__ xt) {
  const long long chunks = (long long)n_bcols * 8;             // 8-neuron chunks per instance
  const long long total = chunks * batch;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(t / chunks);
    const long long c = t - (long long)b * chunks;
    const long long pre0 = c * 8;
    float v[8];
    const float* src = x + (size_t)b * n_pre + pre0;
    if (pre0 + 8 <= n_pre && ((reinterpret_cast<uintptr_t>(src) & 15) == 0)) {
      const float4 lo = *reinterpret_cast<const float4*>(src);
      const float4 hi = *reinterpret_cast<const float4*>(src + 4);
      v[0] = lo.x; v[1] = lo.y; v[2] = lo.z; v[3] = lo.w; v[4] = hi.x; v[5] = hi.y; v[6] = hi.z; v[7] = hi.w;
    } else {
#pragma unroll
      for (int e = 0; e < 8; ++e) v[e] = pre0 + e < n_pre ? src[e] : 0.f;
    }
    const long long tile = c >> 3;
    const int kc = (int)(c & 7);                                 // group of 8 along K
    uint16_t* dst = xt + tile * (long long)batch * kTile + ((b >> 3) * 8 + kc) * 64 + (b & 7) * 8;
    uint4 o;
    o.x = bf16_pair(v[0], v[1]);
    o.y = bf16_pair(v[2], v[3]);
    o.z = bf16_pair(v[4], v[5]);
    o.w = bf16_pair(v[6], v[7]);
    *reinterpret_cast<uint4*>(dst) = o;
  }
}

}  // namespace

extern "C" {

int anb_bsr_tc_pack_x(const float* x, int batch, int n_pre, uint16_t* x_tiles, void* stream) {
  if (!x || !x_tiles || batch <= 0 || batch % 16 != 0 || batch > 256 || n_pre <= 0) return 2;
  const int n_bcols = (n_pre + kTile - 1) / kTile;
  bsr_pack_x_kernel<<<148 * 8, 256, 0, (cudaStream_t)stream>>>(x, batch, n_pre, n_bcols, x_tiles);
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

int anb_bsr_spmm_tc(const int* brow_ptr, const int* bcol, const uint16_t* a_tiles,
                    int n_block_rows, const uint16_t* x_tiles, int batch, float* y, int n_post,
                    int* err, void* stream) {
  if (!brow_ptr || !bcol || !a_tiles || !x_tiles || !y || n_block_rows < 0) return 2;
  if (batch < 16 || batch > 256 || batch % 16 != 0) return 2;
  if (n_block_rows == 0) return 0;
  int cols = 32;
  while (cols < batch) cols <<= 1;
  const size_t smem = (size_t)kStages * (kTileBytes + (size_t)batch * kTile * 2);
  if (cudaFuncSetAttribute(bsr_spmm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return 4;
  bsr_spmm_tc_kernel<<<n_block_rows, 128, smem, (cudaStream_t)stream>>>(
      brow_ptr, bcol, a_tiles, x_tiles, batch, y, n_post, cols, err);
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

int anb_bsr_spmm_simt(const int* brow_ptr, const int* bcol, const uint16_t* a_tiles,
                      int n_block_rows, const uint16_t* x_tiles, int batch, float* y, int n_post,
                      void* stream) {
  if (!brow_ptr || !bcol || !a_tiles || !x_tiles || !y || n_block_rows < 0) return 2;
  if (batch != 64 && batch != 128 && batch != 256) return 2;
  if (n_block_rows == 0) return 0;
  const size_t smem = (size_t)(kTile * kTile + batch * kTile) * 4;
  cudaStream_t st = (cudaStream_t)stream;
#define ANB_SIMT(PER)                                                                              \
  do {                                                                                             \
    if (cudaFuncSetAttribute(bsr_spmm_simt_kernel<PER>,                                           \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) \
      return 4;                                                                                    \
    bsr_spmm_simt_kernel<PER><<<n_block_rows, 256, smem, st>>>(brow_ptr, bcol, a_tiles, x_tiles, \
                                                                 y, n_post);                      \
  } while (0)
  if (batch == 64) ANB_SIMT(16);
  else if (batch == 128) ANB_SIMT(32);
  else ANB_SIMT(64);
#undef ANB_SIMT
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

}  // extern "C"
