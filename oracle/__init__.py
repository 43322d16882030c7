"""CPU oracle for the omegagene hot path -- TEST INFRASTRUCTURE, never the product path."""
