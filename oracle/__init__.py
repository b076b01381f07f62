"""Oracle package: CPU restatement of the reference contraction (test infrastructure only)."""
