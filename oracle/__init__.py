"""CPU oracle of the reference's template-matching path (test infrastructure only).

Nothing in ``kilosort_b200`` imports this package; tests, the smoke check and
the benchmark's CPU-baseline leg use it as the checker.
"""
from . import matching  # noqa: F401
