"""CPU oracle of the reference algorithms (test infrastructure only)."""
