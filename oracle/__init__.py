"""CPU oracle of the PEnGUIn hydro step (test infrastructure only)."""
