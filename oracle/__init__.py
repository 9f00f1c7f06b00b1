"""CPU oracle (test infrastructure only): see ps3d_oracle.cpp."""
