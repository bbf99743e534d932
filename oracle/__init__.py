"""The oracle of the CUDA step -- test infrastructure only (see oracle.py)."""
