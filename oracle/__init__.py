"""PMG oracle (test infrastructure): see oracle/oracle.py."""
