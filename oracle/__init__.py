"""CPU checkers for the snc_b200 backend (test infrastructure only)."""
