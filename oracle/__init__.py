"""CPU oracle (test infrastructure only): C restatement of SciWasm.Sparse's kernels."""
