"""CPU FP64 oracle of the DG operator evaluation (test infrastructure only)."""
