"""CPU oracle package -- test infrastructure only (see sbp_oracle.h)."""
