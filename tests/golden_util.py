"""Loading of the golden fixtures (tests/golden/*.npz)."""
import glob
import os

import numpy as np

from radiance_meshes_b200.camera import make_tcam

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    """The oracle's own fixtures (make_golden.py); the ref_*.npz fixtures hold
    outputs of the reference's code (make_ref_golden.py) and have their own tests."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(p).startswith("ref_"))


def load(name):
    z = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    tcam = make_tcam(z["cam_world_view"].reshape(4, 4), z["cam_K"].reshape(3, 3), z["cam_cam_pos"],
                     int(z["cam_image_height"]), int(z["cam_image_width"]), int(z["cam_tile_width"]),
                     float(z["cam_min_t"]))
    tcam["tile_height"] = int(z["cam_tile_height"])
    tcam["grid_height"] = int(z["cam_grid_height"])
    tcam["grid_width"] = int(z["cam_grid_width"])
    return z, tcam
