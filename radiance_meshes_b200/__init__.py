"""B200-native (sm_100a) differentiable Delaunay-tetrahedral tile rasterizer.

A drop-in for the render path of Radiance Meshes' ``delaunay_rasterization``
package.  Kernels live in ``lib/librm_b200.so`` (built from ``csrc/`` by
``build.py``) behind the C ABI of ``include/rm_capi.h``; Python code here only
allocates tensors, orchestrates launches and wraps them in autograd Functions.
"""
import sys

__version__ = "0.1.0"


def install_dropin() -> None:
    """Make ``import delaunay_rasterization.internal.*`` resolve to this package's
    drop-in modules (same names and signatures as the reference)."""
    from . import delaunay_rasterization as pkg
    from .delaunay_rasterization import internal
    from .delaunay_rasterization.internal import (alphablend_tiled_slang_interp, render_err, render_grid,
                                                  tile_shader_slang, util)

    sys.modules["delaunay_rasterization"] = pkg
    sys.modules["delaunay_rasterization.internal"] = internal
    sys.modules["delaunay_rasterization.internal.tile_shader_slang"] = tile_shader_slang
    sys.modules["delaunay_rasterization.internal.alphablend_tiled_slang_interp"] = alphablend_tiled_slang_interp
    sys.modules["delaunay_rasterization.internal.render_grid"] = render_grid
    sys.modules["delaunay_rasterization.internal.util"] = util
    sys.modules["delaunay_rasterization.internal.render_err"] = render_err
