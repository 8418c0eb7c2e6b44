import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def cuda_ok():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch

    return torch.device("cuda:0")


_PF_CACHE = {}


@pytest.fixture(scope="session")
def plain_forward_oracle():
    """Oracle lists and FP32/FP64 images of the 4,096-point plain-forward
    workload, per tile size."""
    import numpy as np

    from oracle import oracle as O
    from radiance_meshes_b200 import scenes

    def get(tile):
        if tile not in _PF_CACHE:
            mesh, view = scenes.workload_plain_forward(tile)
            tcam = view.tcam(tile_size=tile)
            L = O.rasterize_lists(mesh.indices, mesh.vertices, tcam)
            jitter = np.full((view.height, view.width, 2), 0.5, np.float32)
            img, dist, nc = O.blend_fwd_f32(L, mesh.indices, mesh.vertices, mesh.cell_values, jitter)
            img64 = O.blend_fwd_f64(L, mesh.indices, mesh.vertices.astype(np.float64),
                                    mesh.cell_values.astype(np.float64), jitter, cut=nc)[0]
            _PF_CACHE[tile] = (mesh, view, L, dict(img=img, dist=dist, nc=nc, img64=img64))
        return _PF_CACHE[tile]

    return get
