"""Checker side of the parity tests (test infrastructure, not product)."""
