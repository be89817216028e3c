"""CPU oracle of the reference MLS-MPM step (test infrastructure only)."""
