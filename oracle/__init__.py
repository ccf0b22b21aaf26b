"""CPU oracle of the lighting hot path (test infrastructure only).

Loaded by tests/, __graft_entry__.smoke() and bench.py (cpu_baseline leg and
the CPU reference arm) as the checker; the product library never uses it.
"""
from .binding import Oracle, OracleScene, build_oracle, f16_bits, f16_from_bits  # noqa: F401
