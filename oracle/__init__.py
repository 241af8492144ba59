"""TEST INFRASTRUCTURE ONLY: CPU oracle and reference-library harness (see oracle.py)."""
