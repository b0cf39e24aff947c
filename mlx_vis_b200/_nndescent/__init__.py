"""NNDescent package."""
