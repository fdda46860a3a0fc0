"""Test infrastructure: CPU oracles for the iterNLM hot path (see oracle/oracle.py).

Nothing in the product package imports this.
"""
