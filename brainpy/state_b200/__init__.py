"""brainpy.state_b200 -- B200-native (sm_100a) network step of brainspike.

Public API mirrors the reference Simulator (create / connect / simulate /
cont) with NEST model, rule and device names; the step runs in libbspk's
CUDA kernels (``_lib``).
"""
from . import units
from .simulator import (LogNormal, Normal, NodeView, SimulationResult, Simulator, Uniform,
                        aeif_cond_alpha, all_to_all, fixed_indegree, iaf_cond_alpha, iaf_cond_exp,
                        iaf_psc_alpha, iaf_psc_exp, iaf_psc_exp_multisynapse, multimeter,
                        one_to_one, poisson_generator,
                        spike_recorder, stdp_synapse, stdp_synapse_hom, stdp_triplet_synapse,
                        voltmeter)

__all__ = ["Simulator", "SimulationResult", "NodeView", "iaf_psc_alpha", "iaf_psc_exp",
           "aeif_cond_alpha", "iaf_cond_exp", "iaf_cond_alpha", "iaf_psc_exp_multisynapse",
           "poisson_generator",
           "spike_recorder", "voltmeter", "multimeter", "all_to_all", "one_to_one",
           "fixed_indegree", "stdp_synapse", "stdp_synapse_hom", "stdp_triplet_synapse",
           "Uniform", "Normal", "LogNormal", "units"]
__version__ = "0.1.0"
