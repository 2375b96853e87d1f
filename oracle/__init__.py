"""CPU oracle for the SFINCS time-stepping path (test infrastructure only)."""
