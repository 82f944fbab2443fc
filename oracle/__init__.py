"""CPU oracle for the time-based power path (test infrastructure only)."""
