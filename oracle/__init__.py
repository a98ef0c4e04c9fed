"""CPU oracle and reference-kernel driver: test infrastructure, not shipped code."""
