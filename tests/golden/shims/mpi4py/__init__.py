"""Size-1 stand-in for mpi4py (test infrastructure): one rank, collectives are copies."""
