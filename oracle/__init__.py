"""CPU oracle for the pm3d path (test infrastructure; never imported by pbh_b200)."""
