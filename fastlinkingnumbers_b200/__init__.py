"""B200 linking-number engine: the Gauss linking integral over every
potentially linked loop pair (direct sum and two-tree Barnes–Hut) as
hand-written sm_100a CUDA behind the C ABI of include/fln.h, with the host
stages (BCC loading, potential-link search, Discretize, certificates) in C++.

Python here is a thin mirror of the reference's interface for tests and
benchmarks; the work runs in libfln.so.
"""
from ._native import FlnError, default_params  # noqa: F401
from .api import (  # noqa: F401
    ComputeLinkingNumberDirectFast,
    ComputeLinkingNumberDirectOneArctanPerPair,
    Engine,
    LearnedCriterion,
    LinkingNumberCertificate,
    Model,
    default_engine,
    learned_options,
)
