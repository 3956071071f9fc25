"""Oracle package: TEST INFRASTRUCTURE ONLY (CPU restatement of the reference's path)."""
