"""Oracle for the CKKS evaluation core (test infrastructure only)."""
