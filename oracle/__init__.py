"""CPU oracle for the NUFFT hot path: test infrastructure, never part of the product path."""
