"""CPU oracle for zoomy_amrex_b200 — TEST INFRASTRUCTURE ONLY (see oracle.py)."""
