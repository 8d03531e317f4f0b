"""State comparison used by the parity tests (the package's own comparison routines)."""
from openphase_b200.compare import compare_states, dense_keys, precision_error  # noqa: F401
