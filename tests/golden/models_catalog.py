"""Neuron and synapse definitions whose parsed form is pinned against the
reference parser (ANNarchy/parser/AnalyseNeuron.py:27,
ANNarchy/parser/AnalyseSynapse.py:34).

Each entry is the keyword arguments of ``Neuron(...)`` / ``Synapse(...)``,
valid for both this package and the reference.
"""
from annarchy_b200.workloads import COBA_EQUATIONS, COBA_PARAMS, COBA_RESET, COBA_SPIKE, COBA_REFRACTORY

NEURONS = {
    "input_rate": dict(parameters="r = 0.0"),
    "leaky_integrator": dict(parameters=dict(tau=10.0),
                             equations="tau*dr/dt + r = sum(exc) : min=0.0"),
    "coba_lif": dict(parameters=dict(COBA_PARAMS), equations=list(COBA_EQUATIONS),
                     spike=COBA_SPIKE, reset=COBA_RESET, refractory=COBA_REFRACTORY),
    "rate_pos": dict(parameters="""
            tau = 10.0
            baseline = 0.0
        """,
                     equations="""
            tau * dmp/dt + mp = sum(exc) - sum(inh) + baseline
            r = pos(mp)
        """),
    "izhikevich": dict(parameters="""
            a = 0.02
            b = 0.2
            c = -65.0
            d = 8.0
            I = 0.0
        """,
                       equations="""
            dv/dt = 0.04 * v^2 + 5.0 * v + 140.0 - u + I + g_exc - g_inh : init=-65.0
            du/dt = a * (b*v - u) : init=-13.0
            g_exc = 0.0
            g_inh = 0.0
        """,
                       spike="v >= 30.0",
                       reset="""
            v = c
            u += d
        """),
    "lif_bounded": dict(parameters="""
            tau_m = 10.0 : population
            E_L = -65.0
            v_th = -50.0
        """,
                        equations="""
            tau_m * dv/dt = E_L - v + g_exc : init=-65.0, max=0.0
            tau_m * dg_exc/dt = -g_exc
        """,
                        spike="v > v_th", reset="v = E_L", refractory=2.0),
    "rate_sigmoid_local_tau": dict(parameters="""
            tau = 20.0 : population
            gain = 1.0
        """,
                                   equations="""
            tau * dmp/dt = -mp + sum(exc) : init = 0.1
            r = 1.0 / (1.0 + exp(-gain*mp)) : max = 1.0
        """),
}

# if-then-else statements (the models of the reference's test_ITE.py)
NEURONS.update({
    "ite_simple": dict(equations="r = if (t is 1): 1.0 else: 0.0"),
    "ite_nested": dict(parameters="state = 1.0", equations="""
            r = if (t <= 5):
                    0
                else:
                    if (t >= 7):
                        2
                    else:
                        1
        """),
    "ite_ode": dict(equations="dr/dt = if t > 5: 1 else: 0"),
    "ite_function": dict(equations="r = ite(t is 1, 1.0, 0.0)"),
    "ite_function_nested": dict(parameters="state = 2.0",
                                equations="r = ite(state >= 2, 2, ite(state == 1, 1, 0))"),
    "ite_function_ode": dict(equations="dr/dt = ite((t > 5) and (t <20), 1, 0)"),
})

# population-wide reductions (the model of the reference's test_GlobalOperations.py)
NEURONS["global_operations"] = dict(parameters="r=0", equations="""
            mean_r = mean(r)
            max_r = max(r)
            min_r = min(r)
            l1 = norm1(r)
            l2 = norm2(r)
        """)

SYNAPSES = {
    "stdp": dict(parameters="""
            tau_plus = 16.8 : projection
            tau_minus = 33.7 : projection
            A_plus = 0.005 : projection
            A_minus = 0.00525 : projection
            w_min = 0.0 : projection
            w_max = 1.0 : projection
        """,
                 equations="""
            tau_plus  * dx/dt = -x : event-driven
            tau_minus * dy/dt = -y : event-driven
        """,
                 pre_spike="""
            g_target += w
            x += A_plus * w_max
            w = clip(w + y, w_min , w_max)
        """,
                 post_spike="""
            y -= A_minus * w_max
            w = clip(w + x, w_min , w_max)
        """),
    "spike_default": dict(pre_spike="g_target += w"),
}

# reductions of the pre- and post-synaptic populations in a learning rule
# (the covariance synapse of the reference's test_RateDelays.py)
SYNAPSES["covariance"] = dict(parameters="tau = 5000.0", equations="""
            tau * dw/dt = (pre.r - mean(pre.r) ) * (post.r - mean(post.r) )
        """)
