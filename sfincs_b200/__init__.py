"""B200-native SFINCS time-stepping core (momentum, continuity, CFL dt, boundary forcing)."""
