/*
 * annarchy_b200 — C ABI of the B200 simulation backend.
 *
 * This library replaces the per-network extension module that the reference
 * simulator generates and loads (ANNarchyWrapper<id>, emitted by
 * ANNarchy/generator/NanoBind/Generator.py:18-434 from the template
 * ANNarchy/generator/NanoBind/BaseTemplate.py:1-45). The reference's Python
 * core drives that module through a small set of calls — create the core,
 * set the device, initialise with dt, upload connectivity, get/set
 * attributes, run(n)/step(), set/get time — and this header provides the
 * same operations with plain pointers, sizes and status codes:
 *
 *   - No exception crosses the boundary: every call returns an anb_status;
 *     anb_last_error() gives the message of the last failure on this thread.
 *   - Populations and projections are not C types here. Every attribute of
 *     a population or projection is a named device array ("pop0__v",
 *     "proj1__w", ...); the host side converts the reference's LIL/CSR
 *     connectivity into the storage format and writes it with
 *     anb_array_write. The generated per-network CUDA module declares one
 *     __constant__ pointer "anb_p_<array name>" per array it uses, and the
 *     library binds those pointers to the arrays.
 *   - The per-step work is a list of kernels from that module (grid engine,
 *     one launch each per step, replayed as a CUDA graph) or one persistent
 *     kernel that runs many steps per launch (local engine).
 *
 * Threading: calls on one network must not overlap. All device work is
 * ordered on the network's stream.
 */
#ifndef ANNARCHY_B200_H
#define ANNARCHY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum anb_status {
  ANB_OK = 0,
  ANB_ERR_ARG = 1,       /* invalid argument or unknown name */
  ANB_ERR_ALLOC = 2,     /* device or host allocation failed */
  ANB_ERR_CUDA = 3,      /* a CUDA runtime/driver call failed */
  ANB_ERR_COMPILE = 4,   /* NVRTC rejected the generated module (log in anb_last_error) */
  ANB_ERR_TIMEOUT = 5,   /* a bounded device-side wait gave up (see anb_device_error) */
  ANB_ERR_STATE = 6      /* call out of order (e.g. run before a module is loaded) */
} anb_status;

typedef struct anb_net anb_net;

/* ---- library ---------------------------------------------------------- */

/* Version of this ABI (increments on incompatible changes). */
int anb_abi_version(void);

/* Message of the last failing call on the calling thread ("" if none). */
const char* anb_last_error(void);

/* Number of visible CUDA devices (0 without a GPU). */
int anb_device_count(int* count);

/* Number of streaming multiprocessors of `device` (sizes the persistent
 * launches of batched instances). No counterpart in the reference. */
int anb_device_sm_count(int device, int* count);

/* ---- network lifetime --------------------------------------------------
 * anb_create replaces pyx_create() plus set_device(int)
 * (ANNarchy/generator/NanoBind/BaseTemplate.py:1-45,
 *  ANNarchy/generator/Template/CUDABaseTemplate.py:97-104);
 * anb_initialize replaces pyx_initialize(double dt)
 * (ANNarchy/generator/Compiler.py:888-905). */
int anb_create(int device, anb_net** out);
int anb_destroy(anb_net* net);
int anb_initialize(anb_net* net, double dt);

/* set_time(long) / get_time() of the generated module: the integer step
 * counter t (simulated time is t*dt). */
int anb_set_time(anb_net* net, int64_t t);
int anb_get_time(anb_net* net, int64_t* t);

/* Use a caller-provided cudaStream_t (NULL: the library's own stream). */
int anb_set_stream(anb_net* net, void* cuda_stream);

/* The stream the network's kernels and copies run on (a cudaStream_t), so
 * that other work can be ordered with them. No counterpart in the reference. */
int anb_get_stream(anb_net* net, void** cuda_stream);

/* ---- named device arrays ------------------------------------------------
 * Replace the per-attribute get/set properties of pop<k>_wrapper and the
 * init_from_lil / get/set_local_attribute_* methods of proj<k>_wrapper
 * (ANNarchy/generator/NanoBind/Population.py:27-54,
 *  ANNarchy/generator/NanoBind/Projection.py:20-179). Arrays are zeroed
 * on creation. Reads and writes are synchronous with the network's stream. */
int anb_array_create(anb_net* net, const char* name, size_t bytes);
int anb_array_free(anb_net* net, const char* name);
int anb_array_write(anb_net* net, const char* name, size_t offset, const void* src, size_t bytes);
int anb_array_read(anb_net* net, const char* name, size_t offset, void* dst, size_t bytes);
int anb_array_fill_zero(anb_net* net, const char* name);
int anb_array_info(anb_net* net, const char* name, void** device_ptr, size_t* bytes);

/* Fill an array with a repeated 1-, 2-, 4-, 8- or 16-byte value. */
int anb_array_fill(anb_net* net, const char* name, const void* value, size_t value_bytes);

/* Strided copy of `count` 4-byte elements between two arrays on the device:
 * element i goes from byte src_offset + i * src_stride of `src` to byte
 * dst_offset + i * dst_stride of `dst` (offsets and strides multiples of 4;
 * bounds checked). Packs and unpacks one field of per-synapse records. No
 * counterpart in the reference. */
int anb_array_copy_strided(anb_net* net, const char* dst, size_t dst_offset, size_t dst_stride,
                           const char* src, size_t src_offset, size_t src_stride, size_t count);

/* ---- device-side connectivity -------------------------------------------
 * Replaces the host construction of a fixed_number_pre projection
 * (ANNarchy/core/ConnectorMethods.py:325-370, ANNarchy/cython_ext/
 * Connector.pyx:347-420) for large projections: creates "<prefix>__post_rank"
 * (post ranks post_base..post_base+n_post-1), "__row_ptr", "__col" and "__w"
 * (weight_bytes 8, 4 or 2 = bfloat16). Every row gets `number` distinct pre
 * ranks, one per equal stratum of [pre_lo, pre_hi), ascending; weights are
 * constant a (weight_kind 0), U[a, b) (1) or N(a, b) (2), drawn from a
 * counter-based hash of `seed`. exclude_self moves a draw equal to the post
 * rank to a neighbour in its stratum. */
int anb_connect_fixed_number_pre(anb_net* net, const char* prefix, int n_post, int post_base,
                                 int pre_lo, int pre_hi, int number, uint64_t seed,
                                 int weight_kind, double a, double b, int weight_bytes,
                                 int exclude_self);
/* As anb_connect_fixed_number_pre for rows row_offset .. row_offset + n_post
 * - 1 of a projection whose rows start at post rank post_base - row_offset:
 * the same synapses the whole projection would get for those rows (the
 * random draws are keyed by the projection's row), so a rank can build its
 * share of rows alone. No counterpart in the reference. */
int anb_connect_fixed_number_pre_rows(anb_net* net, const char* prefix, int n_post, int post_base,
                                      long long row_offset, int pre_lo, int pre_hi, int number,
                                      uint64_t seed, int weight_kind, double a, double b,
                                      int weight_bytes, int exclude_self);

/* Distance-based pattern generated on the device (replaces the host
 * construction of ANNarchy/core/ConnectorMethods.py:144-260 and
 * ANNarchy/cython_ext/Connector.pyx:433-575, a Python loop over all pairs):
 * post neuron r (coordinates post_coords[r * dim ..], normalized as the
 * reference's pattern connectors normalize them) receives pre neuron j
 * (pre_coords[j * dim ..]) with the value amp * exp(-d / den) (kind 0,
 * gaussian: a_pos, den_pos) or a_pos * exp(-d / den_pos) - a_neg * exp(-d /
 * den_neg) (kind 1, difference of Gaussians), d the squared distance summed
 * in float over the dimensions (each term in double), the value rounded to
 * float; the pair is kept when the value (kind 1: its magnitude) exceeds
 * threshold; exclude_self drops j == r. Pre ranks ascend per row. Creates the
 * arrays of anb_connect_fixed_number_pre (post_rank, row_ptr, col, w with
 * weight_bytes 8, 4 or 2) and stores the synapse count in *nnz_out. */
int anb_connect_distance_pattern(anb_net* net, const char* prefix, int kind, int n_post,
                                 const double* post_coords, int n_pre, const double* pre_coords,
                                 int dim, double a_pos, double den_pos, double a_neg,
                                 double den_neg, double threshold, int exclude_self,
                                 int weight_bytes, long long* nnz_out);

/* set_seed(long seed, int num_sources, bool use_seed_seq) of the generated
 * module (ANNarchy/generator/NanoBind/BaseTemplate.py:16, called from
 * ANNarchy/generator/Compiler.py:911-922 and ANNarchy/core/Network.py:673-685):
 * the key of the device's counter-based random draws in equations becomes the
 * two 32-bit halves of `seed` (array "rng_seed"). num_sources and
 * use_seed_seq select the reference's per-thread std::mt19937 seeding and have
 * no effect here (one counter-based stream per neuron and draw). */
int anb_set_seed(anb_net* net, uint64_t seed, int num_sources, int use_seed_seq);

/* Declare a recorded state variable: every `period_steps` steps one record of
 * `values_per_record` values of `value_bytes` bytes (the device ring `ring`).
 * Declaring a ring again updates it. Feeds anb_estimate_record_size. No
 * counterpart in the reference (its recorders are compiled in). */
int anb_record_declare(anb_net* net, const char* ring, int64_t values_per_record, int value_bytes,
                       int64_t period_steps);

/* estimate_record_size(int num_steps) of the generated module
 * (ANNarchy/generator/Template/OpenMPBaseTemplate.py:204-211, called from
 * ANNarchy/core/Simulate.py:275-300): MiB the declared recorded state
 * variables take after nsteps more steps (spike records are not counted, as
 * in the reference). */
int anb_estimate_record_size(anb_net* net, int64_t nsteps, size_t* mib);

/* proj<k>_wrapper.init_from_lil(post_ranks, pre_ranks, w, delays,
 * requires_sorting) of the generated module
 * (ANNarchy/generator/NanoBind/Projection.py:20-60, CSR container
 * ANNarchy/include/CSRMatrix.hpp:142), with the list of lists flattened:
 * dendrite r has post rank post_ranks[r] and the synapses row_begin[r] ..
 * row_begin[r + 1] - 1 of pre_ranks, w (double) and delays (steps; NULL for
 * none). Creates "<prefix>__post_rank", "__row_ptr", "__col" (int32) and
 * "__w" (weight_bytes 8, 4 or 2 = bfloat16, rounded to nearest even), plus
 * "__dly" (int32 per synapse) when the delays differ. requires_sorting orders
 * the dendrites by post rank (stable); the synapses of a dendrite keep their
 * order. Invalid input (descending row_begin, negative ranks) gives
 * ANB_ERR_ARG and creates nothing. *nnz_out receives the synapse count. */
int anb_init_from_lil(anb_net* net, const char* prefix, int n_rows, const int* post_ranks,
                      const int64_t* row_begin, const int* pre_ranks, const double* w,
                      const int* delays, int requires_sorting, int weight_bytes, int64_t* nnz_out);

/* Fixed-probability projection generated on the device (replaces the host
 * construction of ANNarchy/core/ConnectorMethods.py:262-330 and
 * ANNarchy/cython_ext/Connector.pyx:306-345, which build per-post Bernoulli
 * masks as lists of lists): every pair (post_base + row, pre) with pre in
 * [pre_lo, pre_hi) is connected with probability 0 < probability <= 1,
 * sampled by geometric skipping keyed by (seed, row_offset + row), pre ranks
 * ascending per row; exclude_self drops pre == post. Creates the arrays of
 * anb_connect_fixed_number_pre (post_rank, row_ptr, col, w) and stores the
 * number of synapses in *nnz_out. */
int anb_connect_fixed_probability_rows(anb_net* net, const char* prefix, int n_post, int post_base,
                                       long long row_offset, int pre_lo, int pre_hi,
                                       double probability, uint64_t seed, int weight_kind, double a,
                                       double b, int weight_bytes, int exclude_self,
                                       long long* nnz_out);

/* Pre-major view of a projection's CSR arrays (the reference's CSRC,
 * ANNarchy/include/CSRCMatrix.hpp:164-222): "<prefix>__col_ptr" over the n_pre
 * neurons of the pre population, "__post_idx" (post rank of each slot),
 * "__inv_idx" (CSR index of each slot) and, with with_weights, "__w_pre". The
 * order of the slots of one pre neuron is unspecified. */
int anb_csr_to_csc(anb_net* net, const char* prefix, int n_pre, int with_weights);

/* ---- generated module ---------------------------------------------------
 * Compiles CUDA C++ source with NVRTC for sm_100a, loads it and binds its
 * __constant__ pointers named "anb_p_<array>" to the arrays of the same
 * name. `options` is a '\n'-separated list of extra NVRTC options. Replaces
 * the reference's CMake/nvcc build of the generated network
 * (ANNarchy/generator/Compiler.py:496-596). */
int anb_module_load(anb_net* net, const char* source, const char* options);

/* Value of a module-scope constant of the loaded module (a float or double
 * `__constant__` variable named `name`, written in its own precision; a
 * constant no kernel uses may be absent from the module, which is not an
 * error).
 * Replaces the generated module's set_<constant>(double)
 * (ANNarchy/generator/NanoBind/BaseTemplate.py:1-45, core/Constant.py). */
int anb_module_set_constant(anb_net* net, const char* name, double value);

/* Compile-only check of a generated module (no device needed): NVRTC for
 * sm_100a; the compiler log is copied into `log` (may be NULL) and the cubin
 * size into *cubin_bytes. */
int anb_nvrtc_compile(const char* source, const char* options, char* log, size_t log_len,
                      size_t* cubin_bytes);

/* Kernels launched, in order, once per simulation step (grid engine). */
int anb_plan_clear(anb_net* net);
int anb_plan_add(anb_net* net, const char* kernel, unsigned grid, unsigned block,
                 unsigned shared_bytes);
/* As anb_plan_add; consecutive plan entries with the same nonzero `group`
 * may run concurrently (forked onto side streams, joined before the next
 * entry; parallel branches of the step's CUDA graph). For kernels that only
 * touch disjoint data or combine their results with atomics (the reference
 * runs its projections one after another, ANNarchy/generator/Template/
 * OpenMPBaseTemplate.py:225-232). */
int anb_plan_add_concurrent(anb_net* net, const char* kernel, unsigned grid, unsigned block,
                            unsigned shared_bytes, int group);

/* Local engine: one kernel `kernel(long long t0, int nsteps)` that runs
 * nsteps steps per launch (grid CTAs, each owning whole network instances). */
int anb_set_local_kernel(anb_net* net, const char* kernel, unsigned grid, unsigned block,
                         unsigned shared_bytes);

/* Same, launched as thread-block clusters of `cluster` CTAs (1..16; sizes
 * above 8 are non-portable). Fails with ANB_ERR_ARG if such a cluster with
 * this much shared memory cannot be scheduled on the device. */
int anb_set_local_kernel_ex(anb_net* net, const char* kernel, unsigned grid, unsigned block,
                            unsigned shared_bytes, unsigned cluster);

/* Steps per captured CUDA graph in the grid engine (0 = no graph). */
int anb_set_graph_steps(anb_net* net, int steps);

/* Programmatic dependent launch of the grid engine's plan (on by default):
 * a kernel that follows another kernel on the network's stream may be
 * scheduled while that one still runs and waits for it on the device
 * (griddepcontrol.wait at its start), which hides the launch latency between
 * the step's dependent kernels. The reference launches each kernel after the
 * previous one returns (ANNarchy/generator/Template/CUDABaseTemplate.py:
 * 328-630). Every kernel of a module run this way must begin with that wait;
 * the generated ones do. */
int anb_set_pdl(anb_net* net, int on);

/* run(int) and step() of the generated module
 * (ANNarchy/generator/Template/CUDABaseTemplate.py:328-630, called from
 * ANNarchy/core/Simulate.py:76-87). Returns after the work is queued;
 * anb_synchronize waits and reports device-side errors. */
int anb_run(anb_net* net, int64_t nsteps);
int anb_step(anb_net* net);

/* Stop condition of population `pop` for anb_run_until: `kernel` (no
 * parameters, launched with grid x block after a step) writes the device step
 * into the int64 array "stop_flags"[pop] when a neuron satisfies the
 * condition (all_mode 0: the condition holds if any neuron does) or when a
 * neuron fails it (all_mode 1: it holds if none fails). No counterpart in the
 * reference, whose populations compile a stop_condition() method
 * (ANNarchy/generator/Population/CUDAGenerator.py:836-917). */
int anb_set_stop_kernel(anb_net* net, int pop, const char* kernel, unsigned grid, unsigned block,
                        int all_mode);

/* Runs at most `steps` steps and stops after the first step at which the
 * stop conditions of the listed populations hold: all of them (or_and != 0)
 * or any (or_and == 0); populations without a condition are skipped, and a
 * non-empty list with none ends an "and" run after one step. Without any stop
 * condition in the network it runs all steps. *done receives the steps run,
 * *stopped 1 when the conditions ended the run. Replaces the reference's
 * run_until(steps, populations, or_and) -> steps run
 * (ANNarchy/generator/Template/OpenMPBaseTemplate.py:95,367-374;
 * CUDABaseTemplate.py:648-680, SimCore/CUDAGenerator.py:478-493). */
int anb_run_until(anb_net* net, int64_t steps, const int* populations, int n_populations, int or_and,
                  int64_t* done, int* stopped);
int anb_synchronize(anb_net* net);

/* Device-side error word: 0, or the code a kernel wrote when a bounded wait
 * gave up or an index check failed; anb_clear_device_error resets it. */
int anb_device_error(anb_net* net, int* code);
int anb_clear_device_error(anb_net* net);

/* ---- monitors ------------------------------------------------------------
 * Decode recorded spike bitmaps (steps x words_per_step words, bit b of word
 * w = neuron 32*w+b) into (step, rank) pairs sorted by step then rank; the
 * host side of the reference's spike recorder (recording_spike_tpl in
 * ANNarchy/generator/Monitor/BaseTemplates.py). Writes at most `capacity`
 * pairs and returns the total number of spikes. Host memory only. */
/* The same decoding on the device, for the first `steps` rows of the spike
 * ring `array` of `net` (words_per_step words per row, bit b of word w =
 * neuron 32*w+b, bits >= n ignored): writes at most `capacity` (step, rank)
 * pairs, sorted by step then rank, into the host arrays and the total number
 * of spikes into *count. Only the pairs cross the bus, not the bitmaps
 * (the reference copies the recorded spikes to the host every step,
 * ANNarchy/generator/Monitor/CUDATemplates.py:83). */
int anb_monitor_decode(anb_net* net, const char* array, int64_t steps, int64_t words_per_step,
                       int64_t n, int32_t* out_steps, int32_t* out_ranks, int64_t capacity,
                       int64_t* count);

int64_t anb_bitmap_decode(const uint32_t* words, int64_t steps, int64_t words_per_step,
                          int64_t n, int64_t* out_steps, int64_t* out_ranks, int64_t capacity);

/* Host-side reordering of a pre-major synapse list for the batched engine's
 * fast delivery, where lane l of a warp adds the synapses of the aligned group
 * of 4 positions 4l..4l+3 of each 128-position block, one shared-memory atomic
 * instruction per block and component. Within each row r (positions
 * row_ptr[r] .. row_ptr[r+1]-1), the synapses ordered by bank (post rank mod
 * 32) are dealt over those instructions in turn, so that an instruction's
 * atomics fall into distinct banks where the row allows it. Writes
 * perm[q - row_ptr[0]] = the position whose synapse goes to position q. The
 * order of additions within a row is free in this mode (float atomics); the
 * reference delivers a spike's synapses in stored order
 * (ANNarchy/generator/Projection/OpenMP/CSR.py:870-902), which only the exact
 * mode keeps. Host memory only. */
int anb_bank_interleave(const int64_t* row_ptr, int64_t n_rows, const int32_t* post, int64_t* perm);

/* ---- batched weighted sums on the tensor cores --------------------------
 * Y[b][post] += sum_pre W[post][pre] * X[b][pre] for `batch` instances that
 * share a block-sparse weight matrix of dense 64 x 64 bfloat16 tiles (the
 * reference's BSR container, ANNarchy/include/BSRMatrix.hpp:41, whose CUDA
 * weighted sum, ANNarchy/generator/Projection/CUDA/BSR.py:296, handles one
 * instance per launch). All pointers are device pointers; `stream` is a
 * cudaStream_t (NULL: the default stream).
 *   a_tiles   n_blocks tiles of 4096 bfloat16 in the tcgen05 canonical
 *             K-major layout (element (r, k) of a tile at
 *             ((r/8)*8 + k/8)*64 + (r%8)*8 + k%8)
 *   x_tiles   ceil(n_pre/64) tiles of batch*64 bfloat16, same layout with
 *             the instance as row: written by anb_bsr_tc_pack_x from
 *             X (batch x n_pre float, row-major)
 *   y         batch x n_post float, row-major, accumulated into
 * batch: a multiple of 16, at most 256 (64, 128 or 256 for
 * anb_bsr_spmm_simt). anb_bsr_spmm_tc runs on the tensor
 * cores (tcgen05.mma, accumulators in tensor memory; bounded waits report
 * ANB_DEVERR_BARRIER_TIMEOUT in *err); anb_bsr_spmm_simt computes the same on
 * the CUDA cores (the comparison baseline). Return 0, 2 (bad argument) or 4
 * (CUDA error). No counterpart in the reference for the batched form. */
int anb_bsr_tc_pack_x(const float* x, int batch, int n_pre, uint16_t* x_tiles, void* stream);
int anb_bsr_spmm_tc(const int* block_row_ptr, const int* block_col, const uint16_t* a_tiles,
                    int n_block_rows, const uint16_t* x_tiles, int batch, float* y, int n_post,
                    int* err, void* stream);
/* Use the module's persistent kernel `kernel(long long t0, int nsteps)` for
 * every run: one cooperative launch (all CTAs resident, so the kernel may
 * separate the phases of a step with grid-wide barriers, bounded waits that
 * report ANB_DEVERR_BARRIER_TIMEOUT) of as many CTAs of `block` threads as
 * fit on all SMs; *grid_out receives that number. The reference launches one
 * kernel per phase and object every step and copies the spike count to the
 * host in between (ANNarchy/generator/Template/CUDABaseTemplate.py:328-630). */
int anb_set_local_kernel_cooperative(anb_net* net, const char* kernel, unsigned block,
                                     unsigned shared_bytes, unsigned* grid_out);

/* Append to the step plan the batched weighted sums of one rate-coded
 * projection shared by `batch` instances: per step the rates in array
 * x_array (batch x n_pre float, row-major) are packed into bfloat16 tiles
 * ("<prefix>__xt") and "<prefix>__brow", "__bcol", "__tiles" (the weights as
 * 64 x 64 bfloat16 blocks, layout of anb_bsr_spmm_tc) add x W^T into y_array
 * (batch x n_post float). Runs on the network's stream inside the step's
 * CUDA graph; `group` as anb_plan_add_concurrent. Replaces, for a batch of
 * network copies, the per-copy BSR weighted sum of
 * ANNarchy/generator/Projection/CUDA/BSR.py:296-392. */
int anb_plan_add_bsr_tc(anb_net* net, const char* prefix, const char* x_array,
                        const char* y_array, int n_block_rows, int batch, int n_pre, int n_post,
                        int group);

/* Launch shape of anb_bsr_spmm_tc for this process: resident CTAs per SM
 * (1-4), shared-memory stages per CTA (2-12) and consecutive blocks of a row
 * per stage (1-8); 0 keeps the automatic choice (two stages; two blocks per
 * stage up to batch 128, one above; up to three CTAs per SM as shared and
 * tensor memory allow; one CTA with up to four stages of two blocks when two
 * do not fit). A later anb_bsr_spmm_tc returns 2 when the shape does not fit
 * its batch (stages above 200 KB in all, or more than 512 tensor-memory
 * columns per SM). Returns 0 or 2. For tuning; no counterpart in the
 * reference. */
int anb_bsr_spmm_tc_shape(int ctas_per_sm, int stages, int group);

/* L2 prefetch distance of anb_bsr_spmm_tc for this process: while copying a
 * block, each CTA keeps the weight tiles of its next `blocks` blocks (0-64;
 * 0 = none, default 4) on their way from HBM into L2 with bulk prefetches.
 * Returns 0 or 2. For tuning; no counterpart in the reference. */
int anb_bsr_spmm_tc_prefetch(int blocks);
int anb_bsr_spmm_simt(const int* block_row_ptr, const int* block_col, const uint16_t* a_tiles,
                      int n_block_rows, const uint16_t* x_tiles, int batch, float* y, int n_post,
                      void* stream);

/* ---- per-kernel timing (CUDA events around every launch; no graphs) -----
 * anb_flush_l2 reads a buffer twice the size of the L2 cache (allocated and
 * filled on first use) on the network's stream, so that the next kernel
 * starts with a cold cache holding no dirty lines; used between timed
 * repetitions. */
int anb_flush_l2(anb_net* net);
/* Cold-read floor: median device time (ms, CUDA events) over `reps` (1-64)
 * repetitions of a streaming read of `bytes` from a fresh buffer, each after
 * anb_flush_l2 (a measuring stick for kernels that must read that many bytes
 * once). No counterpart in the reference. */
int anb_stream_read(anb_net* net, size_t bytes, int reps, double* ms_median);
/* Tile-fill floor: median device time (ms) over `reps` (1-64) launches of
 * `ctas_per_sm` (1-8) CTAs per SM that together copy `copies` tiles of
 * `tile_bytes` (16-65536, a multiple of 16), picked pseudo-randomly from
 * `n_tiles` tiles of an L2-resident buffer, into `stages` (1-16, at most
 * 200 KB in all) shared-memory stages per CTA with bulk copies, each stage
 * with its own issuing thread (after one untimed launch that brings the
 * tiles into L2): the floor of a kernel that stages such tiles through
 * shared memory. No counterpart in the
 * reference. */
int anb_tile_fill(anb_net* net, int n_tiles, int tile_bytes, int copies, int ctas_per_sm, int stages,
                  int reps, double* ms_median);
int anb_kernel_timing(anb_net* net, int enable);
int anb_kernel_time_count(anb_net* net, int* count);
int anb_kernel_time_get(anb_net* net, int index, char* name, size_t name_len,
                        double* total_ms, int64_t* launches);

/* ---- learned storage-format selector -----------------------------------
 * No counterpart in the reference (it uses a fixed rule,
 * ANNarchy/core/Projection.py:691-789). A multilayer perceptron
 * in -> hidden (ReLU) -> hidden (ReLU) -> out maps matrix features to the
 * predicted log10 time of every candidate schedule. Parameters are one float
 * vector W1[hidden][in], b1, W2[hidden][hidden], b2, W3[out][hidden], b3
 * (anb_mlp_param_count floats). All pointers are host pointers; the
 * functions allocate their device buffers themselves. mask[n][out] is 1 for
 * measured targets and 0 otherwise; the loss is the masked mean squared
 * error. Errors: anb_selector_last_error(). */
const char* anb_selector_last_error(void);
size_t anb_mlp_param_count(int in, int hidden, int out);
int anb_mlp_loss_grad(const float* params, const float* x, const float* target, const float* mask,
                      int n, int in, int hidden, int out, float* loss, float* grad);
int anb_mlp_train(float* params, const float* x, const float* target, const float* mask, int n,
                  int in, int hidden, int out, int epochs, float lr, float weight_decay,
                  float* final_loss);
int anb_mlp_predict(const float* params, const float* x, int n, int in, int hidden, int out,
                    float* y);

/* Forward pass of the selector network that allocates no memory; it has no
 * counterpart in the reference. For callers that cannot call cudaMalloc: a
 * simulation loop with real-time deadlines, where the implicit device
 * synchronisation of an allocation would stall it, or a host program whose
 * device memory belongs to another allocator (a pool or a framework's caching
 * allocator). params, x and y are DEVICE pointers owned by the caller;
 * `stream` is a cudaStream_t (NULL: the default stream); the call only
 * queues work. The hidden activations live in a fixed array inside this
 * library (2 MiB on every GPU that loads it, held until exit), so
 * n * hidden must not exceed anb_mlp_noalloc_max_floats() / 2 (ANB_ERR_ARG
 * otherwise). The first call on a device looks up that array's device
 * address; make it before any stream capture. All calls share the array:
 * calls whose work overlaps on the GPU race. */
size_t anb_mlp_noalloc_max_floats(void);
int anb_mlp_predict_noalloc(const float* params, const float* x, int n, int in, int hidden, int out,
                            float* y, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* ANNARCHY_B200_H */
