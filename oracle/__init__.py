"""TEST INFRASTRUCTURE ONLY: CPU oracles for the PR flash (see oracle/oracle.py)."""
