"""FP64 CPU oracle for the batched MMFF optimizer (test infrastructure, never the product path)."""
