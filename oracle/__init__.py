"""CPU oracle of the steady Q1 thermal solve (test infrastructure, not product code)."""
