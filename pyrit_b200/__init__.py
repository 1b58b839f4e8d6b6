"""B200-native (sm_100a) sparse-voxel-DAG build for Pyrit.

The CUDA kernels live in ``libpyrit_b200.so`` behind the C ABI of
``include/pyrit_b200.h``; :mod:`pyrit_b200.gpu_build` mirrors the reference's
``gpu_build`` interface on top of it.
"""
