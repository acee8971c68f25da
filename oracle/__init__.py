"""CPU oracle of the MSLR hot path — test infrastructure only (see mslr_oracle)."""
