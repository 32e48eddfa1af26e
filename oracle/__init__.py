"""CPU oracle for the tridiagonal hot path -- test infrastructure only."""
