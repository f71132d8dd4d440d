"""ORACLE — test infrastructure: the CPU restatement of fenix's step (checker only)."""
