"""Checkers for the CUDA step -- test infrastructure only (see oracle.py)."""
