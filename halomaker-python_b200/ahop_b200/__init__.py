"""ahop_b200: B200-native AdaptaHOP halo finder and batched halo properties.

Public entry points
  * ``compute_adaptahop.neikdtree`` -- drop-in for the reference's f2py module
    (src/compute_neiKDtree_mod.py:36);
  * ``ahop_b200.finder`` -- the same pipeline on numpy or device arrays, with
    stage timings and stage views for parity checks;
  * ``ahop_b200.synthetic`` -- seeded synthetic particle sets.
"""
from ._lib import AhopError, lib  # noqa: F401

__all__ = ["AhopError", "lib"]
