"""ORACLE / TEST INFRASTRUCTURE ONLY: CPU checkers of the wave solver's time stepping."""
