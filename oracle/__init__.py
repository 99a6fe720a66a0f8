"""TEST INFRASTRUCTURE ONLY: the CPU oracle (see oracle/oracle.py)."""
