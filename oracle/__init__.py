"""CPU oracle (test infrastructure only): restatements of REST's RI J/K path.

Nothing in the product package imports this directory; it is the checker.
"""
