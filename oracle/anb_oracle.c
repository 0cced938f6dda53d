/*
 * CPU oracle — TEST INFRASTRUCTURE ONLY.
 *
 * A C restatement of the reference simulator's CPU step for the model
 * families of the benchmark configurations, used by the test suite to check
 * the CUDA backend, by __graft_entry__.smoke() as the checker, and by
 * bench.py as the timed CPU baseline. Nothing in the backend calls it.
 *
 * It restates, in the reference's operation order and with IEEE-754 double
 * arithmetic (build with -ffp-contract=off so no multiply-add is fused):
 *
 *  - the step order of the generated core (ANNarchy/generator/Template/
 *    OpenMPBaseTemplate.py:131-484): zero rate sums -> compute_psp of every
 *    projection (spikes of the previous step) -> neuron update -> spike
 *    gather (ascending ranks) -> post_event of plastic projections -> t++;
 *  - the rate-coded weighted sum of a CSR projection, one sequential sum per
 *    row in ascending pre rank, then `_sum[post] += sum`
 *    (ANNarchy/generator/Projection/OpenMP/CSR.py:177-253);
 *  - event-driven transmission: for every spiking pre neuron in ascending
 *    rank, for its synapses in ascending post rank, `g[post] += w`
 *    (OpenMP/CSR.py:870-902), with the STDP pre-spike statements inlined
 *    (ANNarchy/generator/Projection/OpenMPGenerator.py:910-1100) and the
 *    post-spike statements of post_event (OpenMP/CSR.py:903-922);
 *  - the neuron updates emitted for the leaky integrator
 *    "tau*dr/dt + r = sum(exc) : min=0.0" and for the conductance-based LIF
 *    of the spiking configurations, with the refractory mask of
 *    ANNarchy/generator/Population/OpenMPGenerator.py:870-998 and the spike
 *    gather of :999-1237; refractory steps are int(refractory_ms / dt)
 *    (ANNarchy/core/Population.py:659-690);
 *  - synaptic delays (ANNarchy/generator/Population/SingleThreadGenerator.py
 *    :370-445, SingleThreadTemplates.py:182-212; Projection/
 *    SingleThreadGenerator.py:1186-1195; SingleThread/LIL.py:915-969): a
 *    population keeps the outputs of its last max_delay steps; a rate-coded
 *    projection with delay d reads the rates of step t - d (the history
 *    starts filled with the initial rates); a spiking projection with
 *    uniform delay d propagates the spike list of step t - d; with one delay
 *    per synapse a post neuron receives the spikes by emission step
 *    ascending, then pre rank ascending.
 *
 * Parity pinned against golden fixtures produced by running the reference
 * itself (tests/golden/make_golden.py).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_CLIP(x, a, b) ((x) < (a) ? (a) : ((x) > (b) ? (b) : (x)))

int orc_version(void) { return 2; }

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* rate-coded: leaky integrators fed by CSR projections                      */
/* ------------------------------------------------------------------------ */

/* One rate-coded projection into the integrator population.
 * rows are post ranks 0..n_post-1; col holds pre ranks of population `pre`
 * (0 = the input population, 1 = the integrator population itself). */
typedef struct {
  int pre;
  const int* row_ptr;
  const int* col;
  const double* w;
  int delay;            /* uniform delay in steps (<= 1: the previous step) */
  const int* syn_delay; /* per-synapse delays in steps (CSR order) or NULL */
} orc_rate_proj;

static int orc_slot(int64_t s, int slots) {
  int64_t m = s % slots;
  return (int)(m < 0 ? m + slots : m);
}

/* Simulates `steps` steps of: input population (constant r_in) and one
 * leaky-integrator population of n_out neurons with a single target "exc".
 * r (n_out) is the state (in/out). If r_trace != NULL it receives r after
 * every step (steps x n_out). threads > 1 uses OpenMP like the reference's
 * OpenMP paradigm (rows and neurons split across threads; results are
 * identical to one thread). */
int orc_rate_run(int n_in, int n_out, const double* r_in, double* r, int nproj,
                 const orc_rate_proj* projs, double tau, double dt, double r_min, int steps,
                 double* r_trace, int threads) {
  double* sum = (double*)calloc((size_t)n_out, sizeof(double));
  double* r_prev = (double*)malloc(sizeof(double) * (size_t)n_out);
  /* history of the integrators' rates: slot t % slots holds step t, every
   * slot starting at the initial rates (the input population is constant) */
  int slots = 1;
  for (int p = 0; p < nproj; ++p) {
    if (projs[p].delay > slots) slots = projs[p].delay;
    if (projs[p].syn_delay)
      for (int j = 0; j < projs[p].row_ptr[n_out]; ++j)
        if (projs[p].syn_delay[j] > slots) slots = projs[p].syn_delay[j];
  }
  double* hist = (double*)malloc(sizeof(double) * (size_t)n_out * (size_t)slots);
  if (!sum || !r_prev || !hist) {
    free(sum);
    free(r_prev);
    free(hist);
    return 1;
  }
  for (int q = 0; q < slots; ++q) memcpy(hist + (size_t)q * n_out, r, sizeof(double) * (size_t)n_out);
#ifdef _OPENMP
  if (threads < 1) threads = 1;
#endif
  for (int t = 0; t < steps; ++t) {
    /* the reference reads r of the integrators as it is before this step's update */
    memcpy(r_prev, r, sizeof(double) * (size_t)n_out);
#pragma omp parallel num_threads(threads)
    {
#pragma omp for schedule(static)
      for (int i = 0; i < n_out; ++i) sum[i] = 0.0;
      for (int p = 0; p < nproj; ++p) {
        const orc_rate_proj* pj = &projs[p];
        const int d = pj->delay > 1 ? pj->delay : 1;
        const double* pre_r = pj->pre == 0 ? r_in
                              : (d > 1 ? hist + (size_t)orc_slot(t - d, slots) * n_out : r_prev);
#pragma omp for schedule(static)
        for (int i = 0; i < n_out; ++i) {
          double s = 0.0;
          if (pj->syn_delay && pj->pre != 0) {
            for (int j = pj->row_ptr[i]; j < pj->row_ptr[i + 1]; ++j)
              s += hist[(size_t)orc_slot(t - pj->syn_delay[j], slots) * n_out + pj->col[j]] * pj->w[j];
          } else {
            for (int j = pj->row_ptr[i]; j < pj->row_ptr[i + 1]; ++j) s += pre_r[pj->col[j]] * pj->w[j];
          }
          sum[i] += s;
        }
      }
#pragma omp for schedule(static)
      for (int i = 0; i < n_out; ++i) {
        double _r = (sum[i] - r[i]) / tau;
        r[i] += dt * _r;
        if (r[i] < r_min) r[i] = r_min;
      }
    }
    memcpy(hist + (size_t)orc_slot(t, slots) * n_out, r, sizeof(double) * (size_t)n_out);
    if (r_trace) memcpy(r_trace + (size_t)t * n_out, r, sizeof(double) * (size_t)n_out);
  }
  free(sum);
  free(r_prev);
  free(hist);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* spiking: conductance-based LIF population with event-driven projections   */
/* ------------------------------------------------------------------------ */

typedef struct {
  double El, Vr, Erev_exc, Erev_inh, Vt, tau, tau_exc, tau_inh, I;
} orc_coba_params;

typedef struct {
  double tau_plus, tau_minus, A_plus, A_minus, w_min, w_max;
} orc_stdp_params;

/* One spiking projection within a population of n neurons.
 * CSR part (post-major): rows r = 0..n_rows-1 are post ranks post_rank[r];
 *   row_ptr/col: col = pre rank (population rank), ascending in each row.
 * Column view for propagation: for every pre rank p in 0..n-1,
 *   col_ptr[p]..col_ptr[p+1] lists (row_idx = row, inv_idx = synapse index
 *   into the CSR arrays) in ascending row order.
 * target: 0 -> g_exc, 1 -> g_inh. With stdp != NULL the projection is
 * plastic and x, y, last_event (per synapse, CSR order) are its traces. */
typedef struct {
  int n_rows;
  const int* post_rank;
  const int* row_ptr;
  const int* col;
  double* w;
  const int* col_ptr;
  const int* row_idx;
  const int* inv_idx;
  int target;
  const orc_stdp_params* stdp;
  double* x;
  double* y;
  int64_t* last_event;
  int delay;            /* uniform delay in steps (<= 1: the previous step) */
  const int* syn_delay; /* per-synapse delays in steps (CSR order) or NULL */
} orc_spike_proj;

/* Simulates `steps` steps starting at time step t0. State arrays (length n)
 * are in/out. Every spike is appended to (spike_t, spike_i) up to
 * max_spikes entries; *n_spikes receives the total number of spikes (which
 * may exceed max_spikes). `spiked`/`n_spiked` carry the spike list of the
 * previous step in and the last step's list out (length n). */
int orc_coba_run(int n, const orc_coba_params* prm, int refractory_steps, double dt, int64_t t0,
                 int steps, double* v, double* g_exc, double* g_inh, int* refractory_remaining,
                 int64_t* last_spike, int nproj, const orc_spike_proj* projs, int* spiked,
                 int* n_spiked, int32_t* spike_t, int32_t* spike_i, int64_t max_spikes,
                 int64_t* n_spikes, int threads) {
  short* in_ref = (short*)malloc(sizeof(short) * (size_t)n);
  int* row_of = NULL;
  /* spike lists of the last `slots` steps (slot s % slots holds step s);
   * the step before t0 is the list passed in, older steps had no spikes */
  int slots = 1;
  for (int p = 0; p < nproj; ++p) {
    if (projs[p].delay > slots) slots = projs[p].delay;
    if (projs[p].syn_delay)
      for (int j = 0; j < projs[p].row_ptr[projs[p].n_rows]; ++j)
        if (projs[p].syn_delay[j] > slots) slots = projs[p].syn_delay[j];
  }
  int* hist = (int*)malloc(sizeof(int) * (size_t)n * (size_t)slots);
  int* hist_n = (int*)calloc((size_t)slots, sizeof(int));
  if (!in_ref || !hist || !hist_n) {
    free(in_ref);
    free(hist);
    free(hist_n);
    return 1;
  }
  {
    const int q = orc_slot(t0 - 1, slots);
    hist_n[q] = *n_spiked;
    memcpy(hist + (size_t)q * n, spiked, sizeof(int) * (size_t)(*n_spiked));
  }
  int64_t total = 0;
  int ns = *n_spiked;
#ifdef _OPENMP
  if (threads < 1) threads = 1;
#else
  (void)threads;
#endif
  /* post rank -> row index for plastic projections (the reference searches post_rank) */
  int any_plastic = 0;
  for (int p = 0; p < nproj; ++p) any_plastic |= projs[p].stdp != NULL;
  if (any_plastic) {
    row_of = (int*)malloc(sizeof(int) * (size_t)n * (size_t)nproj);
    if (!row_of) {
      free(in_ref);
      free(hist);
      free(hist_n);
      return 1;
    }
    for (int p = 0; p < nproj; ++p) {
      for (int i = 0; i < n; ++i) row_of[(size_t)p * n + i] = -1;
      for (int r = 0; r < projs[p].n_rows; ++r) row_of[(size_t)p * n + projs[p].post_rank[r]] = r;
    }
  }
  for (int s = 0; s < steps; ++s) {
    const int64_t t = t0 + s;
    /* compute_psp: propagate the (delayed) spikes, projection by projection */
    for (int p = 0; p < nproj; ++p) {
      const orc_spike_proj* pj = &projs[p];
      double* g = pj->target == 0 ? g_exc : g_inh;
      if (pj->syn_delay) {
        /* emission step ascending, spikes ascending, synapses whose delay
         * brings that step's spike to this step */
        for (int64_t s0 = t - slots; s0 < t; ++s0) {
          const int q = orc_slot(s0, slots);
          const int* lst = hist + (size_t)q * n;
          for (int k = 0; k < hist_n[q]; ++k) {
            const int pre = lst[k];
            for (int syn = pj->col_ptr[pre]; syn < pj->col_ptr[pre + 1]; ++syn) {
              const int j = pj->inv_idx[syn];
              if ((int64_t)pj->syn_delay[j] == t - s0) g[pj->post_rank[pj->row_idx[syn]]] += pj->w[j];
            }
          }
        }
        continue;
      }
      const int dq = orc_slot(t - (pj->delay > 1 ? pj->delay : 1), slots);
      const int* lst = hist + (size_t)dq * n;
      for (int k = 0; k < hist_n[dq]; ++k) {
        const int pre = lst[k];
        const int beg = pj->col_ptr[pre], end = pj->col_ptr[pre + 1];
        if (!pj->stdp) {
#pragma omp parallel for num_threads(threads) schedule(static) if (end - beg > 4096)
          for (int syn = beg; syn < end; ++syn) g[pj->post_rank[pj->row_idx[syn]]] += pj->w[pj->inv_idx[syn]];
        } else {
          const orc_stdp_params* sp = pj->stdp;
          for (int syn = beg; syn < end; ++syn) {
            const int j = pj->inv_idx[syn];
            pj->x[j] *= exp(dt * (double)(pj->last_event[j] - (t - 1)) / (sp->tau_plus));
            pj->y[j] *= exp(dt * (double)(pj->last_event[j] - (t - 1)) / (sp->tau_minus));
            pj->last_event[j] = t;
            g[pj->post_rank[pj->row_idx[syn]]] += pj->w[j];
            pj->x[j] += sp->A_plus * sp->w_max;
            pj->w[j] = ORC_CLIP(pj->w[j] + pj->y[j], sp->w_min, sp->w_max);
          }
        }
      }
    }
    /* neuron update */
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int i = 0; i < n; ++i) in_ref[i] = (refractory_remaining[i] > 0) ? 0 : 1;
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int i = 0; i < n; ++i) {
      double _v = (prm->El + prm->Erev_exc * g_exc[i] + prm->Erev_inh * g_inh[i] + prm->I -
                   g_exc[i] * v[i] - g_inh[i] * v[i] - v[i]) / prm->tau;
      double _g_exc = -g_exc[i] / prm->tau_exc;
      double _g_inh = -g_inh[i] / prm->tau_inh;
      v[i] += dt * _v * in_ref[i];
      g_exc[i] += dt * _g_exc;
      g_inh[i] += dt * _g_inh;
      refractory_remaining[i] -= (1 - in_ref[i]);
    }
    /* spike gather, ascending ranks, into this step's slot */
    ns = 0;
    int* cur = hist + (size_t)orc_slot(t, slots) * n;
    for (int i = 0; i < n; ++i) {
      if (in_ref[i] == 0) continue;
      if (v[i] > prm->Vt) {
        v[i] = prm->Vr;
        cur[ns++] = i;
        last_spike[i] = t;
        refractory_remaining[i] = refractory_steps;
        if (total < max_spikes) {
          spike_t[total] = (int32_t)t;
          spike_i[total] = i;
        }
        ++total;
      }
    }
    hist_n[orc_slot(t, slots)] = ns;
    /* post_event of plastic projections */
    for (int p = 0; p < nproj; ++p) {
      const orc_spike_proj* pj = &projs[p];
      if (!pj->stdp) continue;
      const orc_stdp_params* sp = pj->stdp;
      for (int k = 0; k < ns; ++k) {
        const int r = row_of[(size_t)p * n + cur[k]];
        if (r < 0) continue;
        for (int j = pj->row_ptr[r]; j < pj->row_ptr[r + 1]; ++j) {
          pj->x[j] *= exp(dt * (double)(pj->last_event[j] - (t)) / (sp->tau_plus));
          pj->y[j] *= exp(dt * (double)(pj->last_event[j] - (t)) / (sp->tau_minus));
          pj->last_event[j] = t;
          pj->y[j] -= sp->A_minus * sp->w_max;
          pj->w[j] = ORC_CLIP(pj->w[j] + pj->x[j], sp->w_min, sp->w_max);
        }
      }
    }
  }
  {
    const int q = orc_slot(t0 + steps - 1, slots);
    *n_spiked = steps > 0 ? hist_n[q] : *n_spiked;
    if (steps > 0) memcpy(spiked, hist + (size_t)q * n, sizeof(int) * (size_t)hist_n[q]);
  }
  (void)ns;
  *n_spikes = total;
  free(in_ref);
  free(row_of);
  free(hist);
  free(hist_n);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* single operations (used by tests of individual kernels)                    */
/* ------------------------------------------------------------------------ */

/* sum[i] (+)= sequential row sum of w*x over row i of a CSR matrix. */
void orc_csr_rowsum(int n_rows, const int64_t* row_ptr, const int* col, const double* w,
                    const double* x, double* sum, int accumulate) {
  for (int i = 0; i < n_rows; ++i) {
    double s = 0.0;
    for (int64_t j = row_ptr[i]; j < row_ptr[i + 1]; ++j) s += x[col[j]] * w[j];
    sum[i] = accumulate ? sum[i] + s : s;
  }
}

/* ------------------------------------------------------------------------ */
/* Poisson populations (ANNarchy/inputs/PoissonPopulation.py:100-202)        */
/* ------------------------------------------------------------------------ */

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): the backend's generator
 * for random distributions in equations; counter (index, step low, step
 * high, stream), key (seed0, seed1). */
static void orc_philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0, n1 = (uint32_t)p1;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1, n3 = (uint32_t)p0;
    c[0] = n0;
    c[1] = n1;
    c[2] = n2;
    c[3] = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

/* Simulates `steps` steps of n Poisson neurons (no refractory period) in
 * double precision: every step p = 1000 * u / dt with u the 53-bit uniform
 * of draw (seed, stream, t, i), spike when p < rates[i]. Spikes are
 * appended to (spike_t, spike_i) up to max_spikes; returns the total. */
int64_t orc_poisson_run(int n, const double* rates, double dt, const uint32_t* seed, uint32_t stream,
                        int64_t t0, int steps, int32_t* spike_t, int32_t* spike_i, int64_t max_spikes) {
  int64_t total = 0;
  for (int s = 0; s < steps; ++s) {
    const int64_t t = t0 + s;
    for (int i = 0; i < n; ++i) {
      uint32_t c[4] = {(uint32_t)i, (uint32_t)t, (uint32_t)((uint64_t)t >> 32), stream};
      orc_philox(c, seed[0], seed[1]);
      const double u = (double)(((uint64_t)(c[0] >> 6) << 27) | (c[1] >> 5)) * (1.0 / 9007199254740992.0);
      const double rand_0 = 0.0 + (1.0 - 0.0) * u;
      const double p = 1000.0 * rand_0 / dt;
      if (p < rates[i]) {
        if (total < max_spikes) {
          spike_t[total] = (int32_t)t;
          spike_i[total] = i;
        }
        ++total;
      }
    }
  }
  return total;
}
