"""CPU oracle (test infrastructure only): see ``oracle/kennett_oracle.py``."""
