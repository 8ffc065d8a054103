"""CPU oracle for the lattice Monte Carlo hot path (test infrastructure only)."""
