"""import-only stub (point-group symmetry is outside the stand-in)."""
