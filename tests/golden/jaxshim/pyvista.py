"""Rendering is not used by the fixtures."""
