"""Builds the parts of the reference that compile here, unchanged, as
test-only oracles (outputs under oracle/_ref/, which git ignores but the
GPU box receives with the tree).

  sort_by_keys   delaunay_rasterization/internal/sort_by_keys/sort_by_keys.cu,
                 the reference's CUB radix-sort wrapper (a torch extension:
                 cub::DeviceRadixSort::SortPairs on key bits
                 [0, 32 + highest_tile_id_msb)), compiled from its file in the
                 reference tree for sm_100a.  The GPU tests compare
                 rm_sort_pairs with it bit for bit.

Nothing of the product imports this; the reference tree is read only here,
at build time, and never on the GPU box.

    python oracle/build_ref.py [--reference /path/to/reference]
"""
from __future__ import annotations

import argparse
import importlib.machinery
import importlib.util
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
SORT_SRC = os.path.join("delaunay_rasterization", "internal", "sort_by_keys", "sort_by_keys.cu")
SORT_SO = os.path.join(REF_DIR, "sort_by_keys", "sort_by_keys.so")


def build_sort(reference: str, verbose: bool = False) -> str:
    """Compile the reference's sort_by_keys.cu into oracle/_ref/sort_by_keys/."""
    src = os.path.join(reference, SORT_SRC)
    if not os.path.exists(src):
        raise FileNotFoundError(src)
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0a")
    from torch.utils import cpp_extension

    out_dir = os.path.dirname(SORT_SO)
    os.makedirs(out_dir, exist_ok=True)
    if os.path.exists(SORT_SO) and os.path.getmtime(SORT_SO) >= os.path.getmtime(src):
        return SORT_SO
    # compile and link only (no import: this machine may have no GPU)
    cpp_extension.load(name="sort_by_keys", sources=[src], build_directory=out_dir, verbose=verbose,
                       is_python_module=False, is_standalone=False)
    return SORT_SO


def load_sort():
    """The reference's sort_by_keys module (sort_by_keys(keys, values, msb)),
    or None when it was not built."""
    if not os.path.exists(SORT_SO):
        return None
    loader = importlib.machinery.ExtensionFileLoader("sort_by_keys", SORT_SO)
    spec = importlib.util.spec_from_loader("sort_by_keys", loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("RM_REFERENCE_TREE", "/root/reference"))
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build_sort(a.reference, a.verbose))


if __name__ == "__main__":
    sys.exit(main())
