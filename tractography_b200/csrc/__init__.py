"""CUDA sources of libtg_b200.so and the SH-table generator."""
