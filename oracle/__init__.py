"""CPU oracle of the forward-model hot path (test infrastructure only)."""
