"""CPU FP64 oracle (test infrastructure only; see epb_oracle.py)."""
