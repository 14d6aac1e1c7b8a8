"""SciWasm namespace package: `sciwasm.sparse_b200` is the B200 sparse hot path."""
