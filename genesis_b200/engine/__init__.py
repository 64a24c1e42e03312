"""Scene / Simulator / MPMSolver facade over the CUDA runtime."""
