"""CPU oracle of the explicit MLS-MPM substep (test infrastructure only)."""
