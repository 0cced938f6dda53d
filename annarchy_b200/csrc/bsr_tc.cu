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
// Kernel bsr_spmm_tc_kernel (persistent: up to three CTAs per SM, each taking
// block rows blockIdx.x, blockIdx.x + gridDim.x, ...), six warps with fixed
// roles:
//   warp 4 streams the CTA's rows through a ring of shared-memory stages of
//     GROUP consecutive blocks of one row: lane 0 copies the group's weight
//     tiles (contiguous, 8 KB each) in one bulk copy, lane i the batch x 64
//     rate tile of the group's i-th block column (cp.async.bulk completing on
//     the stage's mbarrier; no multicast);
//   warp 5 (one thread) issues the products of a stage (4 per block, K = 16
//     each) into one of two accumulators in tensor memory (rows alternate
//     between them), releases the stage with tcgen05.commit and, after a
//     row's last stage, commits the accumulator to the epilogue;
//   warps 0-3 read the accumulator with tcgen05.ld (warp w reads TMEM lanes
//     32w..32w+31), release it and add it into Y, while the products of the
//     next row run in the other accumulator.
// Two orientations of the product:
//   batch a multiple of 128: D (batch x 64) = X_tile (A, M = 128 per product)
//     x W_tile^T (B, N = 64), accumulator lane = instance, column = post row;
//   otherwise: D (64 x batch) = W_tile (A, M = 64) x X_tile^T (B, N = batch),
//     lane (m % 16) + 32 (m / 16) = post row m, column = instance.
// Every mbarrier wait is bounded and also gives up once another role has
// reported a timeout; the CTA then waits (bounded) for its outstanding copies
// and products, frees its tensor memory and returns.
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
constexpr int kMaxStages = 12;
constexpr unsigned kTileBytes = kTile * kTile * 2;   // 8 KB of bf16
constexpr int kWaitTries = 1 << 22;
constexpr int kThreads = 192;             // warps 0-3 epilogue, 4 copies, 5 products
constexpr int kRowCache = 512;            // block-row ranges held in shared memory

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

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("{ .reg .b64 st; mbarrier.arrive.shared::cta.b64 st, [%0]; }" ::"r"(smem_u32(bar))
               : "memory");
}

// Bounded wait for the phase of parity `parity`; false on timeout or when
// *abort is set (checked every 64 polls).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, const volatile int* abort) {
  const unsigned b = smem_u32(bar);
  unsigned done = 0;
  for (int it = 0; it < kWaitTries && !done; ++it) {
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done) : "r"(b), "r"(parity) : "memory");
    if (!done && (it & 63) == 63 && abort && *abort) return false;
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

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// y[0..15] += r[0..15] for 16 consecutive floats (vector access when aligned);
// all loads are issued before the tensor-memory read completes.
__device__ __forceinline__ void add16_contiguous(float* y, uint32_t taddr, bool vec, int valid) {
  float old[16];
  uint32_t r[16];
  if (vec) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float4 o = reinterpret_cast<const float4*>(y)[q];
      old[4 * q] = o.x; old[4 * q + 1] = o.y; old[4 * q + 2] = o.z; old[4 * q + 3] = o.w;
    }
  } else {
#pragma unroll
    for (int j = 0; j < 16; ++j) old[j] = j < valid ? y[j] : 0.f;
  }
  tmem_ld16(taddr, r);
  if (vec) {
#pragma unroll
    for (int q = 0; q < 4; ++q)
      reinterpret_cast<float4*>(y)[q] =
          make_float4(old[4 * q] + __uint_as_float(r[4 * q]), old[4 * q + 1] + __uint_as_float(r[4 * q + 1]),
                      old[4 * q + 2] + __uint_as_float(r[4 * q + 2]),
                      old[4 * q + 3] + __uint_as_float(r[4 * q + 3]));
  } else {
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (j < valid) y[j] = old[j] + __uint_as_float(r[j]);
  }
}

// Block range of the CTA's i-th block row br (from shared memory when cached).
__device__ __forceinline__ int2 tc_row(const int2* rows_s, const int* brow_ptr, int i, int br) {
  return i < kRowCache ? rows_s[i] : make_int2(brow_ptr[br], brow_ptr[br + 1]);
}

__global__ void __launch_bounds__(kThreads, 1)
bsr_spmm_tc_kernel(const int* __restrict__ brow_ptr, const int* __restrict__ bcol,
                   const uint16_t* __restrict__ a_tiles, const uint16_t* __restrict__ x_tiles,
                   int n_block_rows, int batch, float* __restrict__ y, int n_post, int stages,
                   int group, int xmajor, int acc_cols, int tmem_cols, int prefetch, int* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t full[kMaxStages], empty[kMaxStages], acc_full[2], acc_empty[2], done;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;
  __shared__ int issued_n, consumed_n, mma_any;
  __shared__ int2 rows_s[kRowCache];       // [beg, end) of the CTA's block rows i = 0, 1, ...
  const unsigned x_bytes = (unsigned)batch * kTile * 2;
  // a stage: `group` weight tiles (consecutive blocks of one row), then their
  // `group` rate tiles
  const unsigned stage_bytes = (unsigned)group * (kTileBytes + x_bytes);
  const unsigned x_off = (unsigned)group * kTileBytes;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(&tmem_base)), "r"(tmem_cols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < stages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&acc_full[a], 1);
      mbar_init(&acc_empty[a], 4);          // one arrival per epilogue warp
    }
    mbar_init(&done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
    issued_n = 0;
    consumed_n = 0;
    mma_any = 0;
  }
  for (int i = threadIdx.x; i < kRowCache; i += kThreads) {
    const int br = blockIdx.x + i * gridDim.x;
    if (br < n_block_rows) rows_s[i] = make_int2(brow_ptr[br], brow_ptr[br + 1]);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = tmem_base;

  if (warp == 4) {
    // the whole warp: lane i fetches the block column of the stage's i-th
    // block (while the stage is still being released) and copies its rate
    // tile; lane 0 copies the stage's weight tiles in one piece
    int s = 0, k = 0;                         // stage, stages filled
    unsigned ph = 0;                          // parity of the stage's current use
    bool ok = true;
    // lane 0 also keeps the weight tiles of the CTA's next `prefetch` blocks
    // on their way into L2 (bulk prefetch), so that their copies into shared
    // memory wait for L2 rather than HBM: cursor (row i, block range
    // [pf_b, pf_e) left in it), blocks prefetched pf_n, blocks copied cp_n
    int pf_i = 0, pf_br = blockIdx.x, pf_b = 0, pf_e = 0, pf_n = 0, cp_n = 0;
    if (lane == 0 && prefetch > 0 && pf_br < n_block_rows) {
      const int2 r0 = tc_row(rows_s, brow_ptr, 0, pf_br);
      pf_b = r0.x;
      pf_e = r0.y;
    }
    for (int i = 0, br = blockIdx.x; br < n_block_rows && ok; ++i, br += gridDim.x) {
      const int2 rr = tc_row(rows_s, brow_ptr, i, br);
      for (int g0 = rr.x; g0 < rr.y; g0 += group) {
        const int gn = rr.y - g0 < group ? rr.y - g0 : group;
        const int bc = lane < gn ? bcol[g0 + lane] : 0;
        if (k >= stages) {
          const bool w = __all_sync(0xffffffffu, mbar_wait(&empty[s], ph ^ 1u, &abort_flag));
          if (!w) {
            if (lane == 0) {
              anb_report(err, ANB_DEVERR_BARRIER_TIMEOUT);
              abort_flag = 1;
            }
            ok = false;
            break;
          }
        }
        unsigned char* st = smem + s * stage_bytes;
        if (lane == 0) mbar_expect_tx(&full[s], (unsigned)gn * (kTileBytes + x_bytes));
        __syncwarp();
        if (lane == 0) bulk_load(st, a_tiles + (size_t)g0 * (kTile * kTile), (unsigned)gn * kTileBytes, &full[s]);
        if (lane < gn) bulk_load(st + x_off + lane * x_bytes, x_tiles + (size_t)bc * batch * kTile, x_bytes, &full[s]);
        if (lane == 0 && prefetch > 0) {
          cp_n += gn;
          while (pf_br < n_block_rows && pf_n < cp_n + prefetch) {
            const int want = min(pf_e - pf_b, cp_n + prefetch - pf_n);
            if (want > 0) {
              asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;"
                           ::"l"(a_tiles + (size_t)pf_b * (kTile * kTile)), "r"((unsigned)want * kTileBytes)
                           : "memory");
              pf_b += want;
              pf_n += want;
            }
            if (pf_b >= pf_e) {               // next row of this CTA
              ++pf_i;
              pf_br += gridDim.x;
              if (pf_br < n_block_rows) {
                const int2 r = tc_row(rows_s, brow_ptr, pf_i, pf_br);
                pf_b = r.x;
                pf_e = r.y;
              }
            }
          }
        }
        ++k;
        if (++s == stages) {
          s = 0;
          ph ^= 1u;
        }
      }
    }
    if (lane == 0) {
      issued_n = k;
      // every stage released by its products before the CTA leaves: the last
      // use of each stage, in fill order
      for (int q = 0; ok && q < (k < stages ? k : stages); ++q) {
        const int kq = k - 1 - q;               // a stage filled kq-th, use kq / stages
        if (!mbar_wait(&empty[kq % stages], (unsigned)(kq / stages) & 1u, &abort_flag)) {
          anb_report(err, ANB_DEVERR_BARRIER_TIMEOUT);
          abort_flag = 1;
          ok = false;
        }
      }
    }
  } else if (warp == 5) {
    if (lane == 0) {
      const uint32_t idesc = xmajor ? instr_desc(128, kTile) : instr_desc(kTile, batch);
      const int halves = xmajor ? batch / 128 : 1;
      // descriptors of the start of shared memory; offsets added in 16-byte units
      const uint64_t d0 = smem_desc(smem_u32(smem), 128, 1024);
      int s = 0, k = 0, t = 0;                // stage, stages consumed, non-empty rows done
      unsigned ph = 0;
      bool ok = true;
      for (int i = 0, br = blockIdx.x; br < n_block_rows && ok; ++i, br += gridDim.x) {
        const int2 rr = tc_row(rows_s, brow_ptr, i, br);
        if (rr.y == rr.x) continue;
        const int a = t & 1, v = t >> 1;
        if (v > 0 && !mbar_wait(&acc_empty[a], (v - 1) & 1, &abort_flag)) {
          anb_report(err, ANB_DEVERR_BARRIER_TIMEOUT);
          abort_flag = 1;
          break;
        }
        tc_fence_after();
        const uint32_t d = tbase + (uint32_t)(a * acc_cols);
        for (int g0 = rr.x; g0 < rr.y; g0 += group) {
          const int gn = rr.y - g0 < group ? rr.y - g0 : group;
          if (!mbar_wait(&full[s], ph, &abort_flag)) {
            anb_report(err, ANB_DEVERR_BARRIER_TIMEOUT);
            abort_flag = 1;
            ok = false;
            break;
          }
          tc_fence_after();
          const uint64_t ws = d0 + ((s * stage_bytes) >> 4);
          const uint64_t xs = ws + (x_off >> 4);
          for (int b = 0; b < gn; ++b) {
            const uint64_t wb = ws + ((b * kTileBytes) >> 4), xb = xs + ((b * x_bytes) >> 4);
            const uint32_t acc0 = (g0 > rr.x || b > 0) ? 1u : 0u;
            if (xmajor) {
              for (int h = 0; h < halves; ++h) {
#pragma unroll
                for (int q = 0; q < kTile / 16; ++q)
                  umma_f16(d + (uint32_t)(h * kTile), xb + h * (16384 >> 4) + q * (256 >> 4), wb + q * (256 >> 4),
                           idesc, (acc0 | q) ? 1u : 0u);
              }
            } else {
#pragma unroll
              for (int q = 0; q < kTile / 16; ++q)
                umma_f16(d, wb + q * (256 >> 4), xb + q * (256 >> 4), idesc, (acc0 | q) ? 1u : 0u);
            }
          }
          mma_any = 1;
          umma_commit(&empty[s]);
          ++k;
          if (++s == stages) {
            s = 0;
            ph ^= 1u;
          }
        }
        if (!ok) break;
        umma_commit(&acc_full[a]);
        ++t;
      }
      consumed_n = k;
      if (mma_any) umma_commit(&done);        // after every issued product
    }
  } else {
    // epilogue warps 0-3
    const bool vec = (n_post & 3) == 0 && (reinterpret_cast<uintptr_t>(y) & 15) == 0;
    int t = 0;
    for (int i = 0, br = blockIdx.x; br < n_block_rows; ++i, br += gridDim.x) {
      const int2 rr = tc_row(rows_s, brow_ptr, i, br);
      if (rr.y == rr.x) continue;
      const int a = t & 1, v = t >> 1;
      const bool ok = __all_sync(0xffffffffu, mbar_wait(&acc_full[a], v & 1, &abort_flag));
      if (!ok) {
        if (lane == 0) {
          anb_report(err, ANB_DEVERR_BARRIER_TIMEOUT);
          abort_flag = 1;
        }
        break;
      }
      tc_fence_after();
      const uint32_t tw = tbase + ((uint32_t)(32 * warp) << 16) + (uint32_t)(a * acc_cols);
      if (xmajor) {
        // lane = instance 32 w + lane (+128 per half); 64 consecutive post rows
        const int r0 = br * kTile;
        const int valid_rows = n_post - r0 < kTile ? n_post - r0 : kTile;
        for (int h = 0; h < batch / 128; ++h) {
          float* yb = y + (size_t)(h * 128 + 32 * warp + lane) * n_post + r0;
#pragma unroll 1
          for (int c0 = 0; c0 < kTile; c0 += 16) {
            const int valid = valid_rows - c0 < 16 ? (valid_rows - c0 > 0 ? valid_rows - c0 : 0) : 16;
            add16_contiguous(yb + c0, tw + (uint32_t)(h * kTile + c0), vec && valid == 16, valid);
          }
        }
      } else {
        // lanes 0-15 of warp w hold post rows 16 w .. 16 w + 15; columns = instances
        const int row = br * kTile + 16 * warp + lane;
        const bool mine = lane < 16 && row < n_post;
        for (int c0 = 0; c0 < batch; c0 += 16) {
          float old[16];
          uint32_t r[16];
          if (mine) {
#pragma unroll
            for (int j = 0; j < 16; ++j) old[j] = y[(size_t)(c0 + j) * n_post + row];
          }
          tmem_ld16(tw + (uint32_t)c0, r);
          if (mine) {
#pragma unroll
            for (int j = 0; j < 16; ++j) y[(size_t)(c0 + j) * n_post + row] = old[j] + __uint_as_float(r[j]);
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[a]);
      ++t;
    }
  }
  __syncthreads();
  if (abort_flag && threadIdx.x == 0) {
    // copies issued but never consumed: wait for them (bounded) before leaving
    for (int k = consumed_n; k < issued_n; ++k) mbar_wait(&full[k % stages], (unsigned)(k / stages) & 1u, nullptr);
  }
  if (mma_any && threadIdx.x == 0 && !mbar_wait(&done, 0, nullptr))
    anb_report(err, ANB_DEVERR_BARRIER_TIMEOUT);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 5) {
    __syncwarp();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(tmem_cols)
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

// launch-shape overrides of anb_bsr_spmm_tc (0 = automatic)
int g_tc_per_sm = 0;
int g_tc_stages = 0;
int g_tc_group = 0;
// L2 prefetch distance of the weight tiles, in blocks (0 = none). On the
// 100k block matrix 4 blocks ahead gained 1-3 % at batches 16-256; 16 or
// more lost 15-40 % (the prefetched tiles crowd the rate tiles out of L2)
int g_tc_prefetch = 4;

}  // namespace

extern "C" {

int anb_bsr_tc_pack_x(const float* x, int batch, int n_pre, uint16_t* x_tiles, void* stream) {
  if (!x || !x_tiles || batch <= 0 || batch % 16 != 0 || batch > 256 || n_pre <= 0) return 2;
  const int n_bcols = (n_pre + kTile - 1) / kTile;
  bsr_pack_x_kernel<<<148 * 8, 256, 0, (cudaStream_t)stream>>>(x, batch, n_pre, n_bcols, x_tiles);
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

int anb_bsr_spmm_tc_shape(int ctas_per_sm, int stages, int group) {
  if (ctas_per_sm < 0 || ctas_per_sm > 4 || stages < 0 || stages == 1 || stages > kMaxStages ||
      group < 0 || group > 8)
    return 2;
  g_tc_per_sm = ctas_per_sm;
  g_tc_stages = stages;
  g_tc_group = group;
  return 0;
}

int anb_bsr_spmm_tc_prefetch(int blocks) {
  if (blocks < 0 || blocks > 64) return 2;
  g_tc_prefetch = blocks;
  return 0;
}

int anb_bsr_spmm_tc(const int* brow_ptr, const int* bcol, const uint16_t* a_tiles,
                    int n_block_rows, const uint16_t* x_tiles, int batch, float* y, int n_post,
                    int* err, void* stream) {
  if (!brow_ptr || !bcol || !a_tiles || !x_tiles || !y || n_block_rows < 0) return 2;
  if (batch < 16 || batch > 256 || batch % 16 != 0) return 2;
  if (n_block_rows == 0) return 0;
  static int sm_count = 0;
  if (sm_count == 0) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return 4;
  }
  // accumulators: two per CTA, a power of two of columns each
  const int xmajor = batch % 128 == 0 ? 1 : 0;
  const int need = xmajor ? kTile * (batch / 128) : batch;
  int acc_cols = 32;
  while (acc_cols < need) acc_cols <<= 1;
  const int tmem_cols = 2 * acc_cols;
  // shape: `group` blocks per stage, `stages` stages, `per_sm` CTAs per SM.
  // Each CTA's copy and product threads spend a few hundred cycles of their
  // own per stage, so several CTAs per SM and two blocks per stage keep HBM
  // busy better than deep rings: two stages, as many CTAs (up to three) as
  // shared and tensor memory allow, else one CTA with up to four stages of
  // two blocks. anb_bsr_spmm_tc_shape overrides the choice.
  const size_t block_bytes = kTileBytes + (size_t)batch * kTile * 2;
  const int tm_limit = 512 / tmem_cols;
  int per_sm = 1, group = 2, stages = 2;
  if (tm_limit >= 2) {
    group = 4 * block_bytes <= (104u << 10) ? 2 : 1;
    per_sm = (int)((222u << 10) / ((size_t)stages * group * block_bytes + (6u << 10)));
    if (per_sm > 3) per_sm = 3;
    if (per_sm > tm_limit) per_sm = tm_limit;
  }
  if (per_sm < 2) {
    per_sm = 1;
    group = 2;
    stages = (int)((200u << 10) / (group * block_bytes));
    if (stages > 4) stages = 4;
  }
  if (g_tc_per_sm > 0) per_sm = g_tc_per_sm;
  if (g_tc_stages > 0) stages = g_tc_stages;
  if (g_tc_group > 0) group = g_tc_group;
  const size_t smem = (size_t)stages * group * block_bytes;
  if (stages < 2 || stages > kMaxStages || group < 1 || group > 8 || smem > (200u << 10) ||
      per_sm * tmem_cols > 512)
    return 2;
  if (cudaFuncSetAttribute(bsr_spmm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return 4;
  const int grid = n_block_rows < per_sm * sm_count ? n_block_rows : per_sm * sm_count;
  bsr_spmm_tc_kernel<<<grid, kThreads, smem, (cudaStream_t)stream>>>(
      brow_ptr, bcol, a_tiles, x_tiles, n_block_rows, batch, y, n_post, stages, group, xmajor,
      acc_cols, tmem_cols, g_tc_prefetch, err);
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
