"""spo_b200: the split-operator propagation step of SPO-DVR on the NVIDIA B200 (sm_100a).

The compute path is the C ABI of include/spo_b200.h (lib/libspo_b200.so); this package is its host
side: the PropagationBackend-shaped wrapper, case bundles and the benchmark's synthetic workloads.
"""

from .backend import B200Backend, Ensemble  # noqa: F401
from .capi import B200Error  # noqa: F401
from .case import CaseBundle  # noqa: F401

__version__ = "0.1.0"
