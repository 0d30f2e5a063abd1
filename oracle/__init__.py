"""CPU oracle of the BEADS hot path (test infrastructure, never shipped)."""
