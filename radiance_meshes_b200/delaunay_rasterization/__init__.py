"""Drop-in replacement of the reference package ``delaunay_rasterization``.

Same module names, classes and call signatures as
``delaunay_rasterization/internal/{tile_shader_slang,alphablend_tiled_slang_interp,
render_grid,util}.py``; the kernels behind them are the sm_100a kernels of
``librm_b200.so``.  ``radiance_meshes_b200.install_dropin()`` registers this
package under the reference's import path.
"""
__version__ = "0.1.0"
