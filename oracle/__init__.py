"""CPU oracle for the K2 evaluator (test infrastructure only; see oracle.py)."""
