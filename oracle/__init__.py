"""Correctness oracle for hmfem's pressure-solve path (test infrastructure
only; never imported by the GPU product path)."""
