"""Parameters of the synthetic-mesh golden case (shared by its generator and tests)."""
N_NODES, SEED, DT = 600, 3, 1800.0
