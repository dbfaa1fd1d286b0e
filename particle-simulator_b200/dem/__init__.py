"""Drop-in, B200-native DEM droplet hot path.

The subpackages mirror ddkx21/particle-simulator's ``dem`` package (same module
paths, class names, constructor arguments and methods); their compute runs in
the CUDA kernels of ``libdem_b200.so`` through the C ABI of ``include/dem_b200.h``.
"""
