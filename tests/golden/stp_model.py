"""Tsodyks-Markram short-term plasticity as a synapse description, shared
by the fixture maker (run on the reference) and the tests (run on this
backend): event-driven recovery x and facilitation u, both updated at each
pre-synaptic spike, the transmission scaled by u * x."""

STP_PARAMETERS = """
    tau_rec = 200.0 : projection
    tau_facil = 50.0 : projection
    U = 0.2
"""
STP_EQUATIONS = """
    dx/dt = (1 - x)/tau_rec : init = 1.0, event-driven
    du/dt = (U - u)/tau_facil : init = 0.2, event-driven
"""
STP_PRE_SPIKE = """
    g_target += w * u * x
    x *= (1 - u)
    u += U * (1 - u)
"""
