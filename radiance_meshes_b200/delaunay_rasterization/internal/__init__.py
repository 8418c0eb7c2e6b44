"""Reference-named modules of the B200 rasterizer (see the package docstring)."""
