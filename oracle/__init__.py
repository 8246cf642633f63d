"""CPU oracle of the WCSPH step (test infrastructure only; see oracle.py)."""
