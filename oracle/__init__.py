"""CPU oracle of the Lambent path-tracing hot path (test infrastructure only)."""
