"""Voxelisation is not used by the fixtures."""
