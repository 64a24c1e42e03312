"""CPU oracle of the MPM substep -- test infrastructure only (see mpm_ref.py)."""
