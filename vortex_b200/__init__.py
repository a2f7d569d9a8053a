"""B200-native vortex-element time step (drop-in for grechkin-pogrebnyakov/vortex).

The product is the C ABI library ``libvortex_b200.so`` (include/vortex_b200.h,
include/vortex_b200_unit1.h) and the ``bin/vortex`` CLI built from csrc/.
``vortex_b200.native`` binds the library for Python callers; ``profiles``
generates and reads body profiles.
"""
__all__ = ["native", "profiles", "build"]
