"""CPU oracle of the render path (test infrastructure only; see oracle.c)."""
