"""The oracle: a CPU restatement of GeometricSolvers.jl's R2 batch, used as the checker by the
tests, the smoke check and bench.py's CPU-baseline leg only."""
