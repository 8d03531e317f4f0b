"""openphase_b200 — B200-native multiphase-field time step of OpenPhase (CUDA sm_100a + C ABI)."""
from ._lib import OpgpuError, device_count, lib  # noqa: F401
