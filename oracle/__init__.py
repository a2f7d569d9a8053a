"""CPU oracle package (test infrastructure only; see vx_oracle.h)."""
