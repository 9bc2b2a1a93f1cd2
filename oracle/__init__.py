"""CPU oracle for the Pearl hot path — test infrastructure only (see pyoracle.py)."""
