"""Test infrastructure only: the CPU checkers (see oracle.py). Not part of the product."""
