"""CPU oracle for the voxelG traversal path (test infrastructure only)."""
