"""Synthetic workloads of the benchmark configurations (meshes, kernels,
loop chains), shared by bench.py and the tests."""
