"""CPU FP64 oracle of the ChiDG linear-solve path (test infrastructure only)."""
