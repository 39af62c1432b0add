"""TEST INFRASTRUCTURE: CPU checkers for the render hot path (see oracle.py).
Never imported by the product package."""
