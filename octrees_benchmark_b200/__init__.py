"""B200-native linear-octree neighbour search (drop-in for the point-cloud
neighbour-search path of derivada/octrees-benchmark).

The compute path is liboctree_b200.so (hand-written sm_100a CUDA behind the C
ABI in include/octree_b200.h); this package holds its sources (csrc/), its
build recipe (build.py), a ctypes binding (capi.py), a Python front end with
the reference's names (linear_octree.py) and the synthetic LiDAR generator
shared by the tests and the benchmark (synth.py).
"""
from .capi import OctError, header_functions, lib  # noqa: F401
from .linear_octree import LinearOctree  # noqa: F401

__all__ = ["LinearOctree", "OctError", "lib", "header_functions"]
