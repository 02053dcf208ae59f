"""B200-native hourly land-surface step of IBIS 3.0: CUDA kernels for sm_100a behind a C ABI, and the Python host side."""
