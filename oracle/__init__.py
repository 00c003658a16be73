"""CPU oracle of the LocVolCalib path -- test infrastructure only (see oracle.py)."""
