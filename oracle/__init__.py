"""CPU checkers for the dyphur frame step (test infrastructure only)."""
