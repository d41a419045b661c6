"""B200-native neural tick for Neural Selection (placeholder, filled below)."""
from . import workloads  # noqa: F401
