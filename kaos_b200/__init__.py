"""kaos_b200 -- B200-native kinetic particle loop of KAOS (Kinetic model of
Auroral ion OutflowS) behind a C-ABI (include/kaos_gpu.h)."""
from .model_input import ModelInput, Tube, VGrid  # noqa: F401

__version__ = "0.1.0"
