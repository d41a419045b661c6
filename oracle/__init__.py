"""ORACLE — test infrastructure: CPU restatement of the reference neural tick,
the reference's own host executor built from its sources, and their drivers."""
