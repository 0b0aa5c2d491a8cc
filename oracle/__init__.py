"""FP64 CPU oracle of the reference's per-step solve (test infrastructure only)."""
