"""CPU checkers for the CUDA hot path — test infrastructure only (see cases.py)."""
