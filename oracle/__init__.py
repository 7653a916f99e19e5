"""CPU oracles of the hot path (test infrastructure only)."""
