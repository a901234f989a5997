"""B200-native refactor-and-solve engine for SPICE MNA matrices.

The product is libluspice_b200.so (host analysis in C/C++, sm_100a kernels,
C-ABI in include/*.h).  This package holds its build script, ctypes
bindings (_lib), a thin Python host wrapper (api) and the seeded synthetic
MNA generators (mna).  Importing the package loads nothing; api calls load
the library and raise if it has not been built.
"""
__all__ = ["api", "mna", "build"]
