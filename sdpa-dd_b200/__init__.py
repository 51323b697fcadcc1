"""sdpa-dd_b200: the SDPA-DD dd Newton hot path on NVIDIA B200 (sm_100a).

The product is the C-ABI library `libsddd.so` (declared in include/sddd.h)
and the `sdpa_dd_b200` command-line driver built from csrc/.  This Python
package only locates and binds them (ctypes) and generates workloads.
"""
