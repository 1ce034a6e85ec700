"""Plotting is not used by the fixtures."""
