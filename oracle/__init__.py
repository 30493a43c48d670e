"""CPU oracle for the CEL solver hot path (test infrastructure only)."""
