"""CPU oracle for the Lenia field update (test infrastructure only)."""
