"""qompsim -- helpers around the qulacs-compatible engine: the seeded
synthetic workloads the engine is measured on (circuits), and the one-rank
driver mode of the reference's run_sim.py (run_sim)."""
