"""Determinant-basis FCI core (link tables, sigma, diagonal, RDMs, Davidson)."""
from . import direct_spin1, davidson  # noqa: F401
