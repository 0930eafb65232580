"""srmg: B200-native FAS multigrid field solve for Steamroller.jl trees.

Python host side of the C-ABI library ``libsrmg.so``: a mirror of the reference's
tree/connectivity types (``tree``), seeded workload generators (``gen``) and the
ctypes binding with the reference's entry-point names (``multigrid``).
"""
