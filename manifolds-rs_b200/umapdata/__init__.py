"""umapdata: inputs of the UMAP layout path that need no GPU library.

Seeded synthetic data of the benchmark workloads' shapes (``synth``) and a
NumPy reader / writer of the kNN cache file format (``knn_cache``; the same
format as ``umapcu_knn_save`` / ``umapcu_knn_load``). Importing this package
loads no native code of the umapcu library, so a process that must not run
the CUDA path (the CPU reference timing, tooling that only prepares inputs)
can use it.
"""
