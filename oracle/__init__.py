"""CPU oracle of the tetrahedral tile rasterizer (test infrastructure only)."""
