"""B200 engine for the orbital-free DFT density solve of PROFESS.

The product is the CUDA library ``_lib/libprofess_b200.so`` (C ABI in
``include/profess_b200.h``); this package holds its ctypes binding
(``native``), the cell set-up on top of it (``cell``), the synthetic
workloads (``workloads``, ``recpot``) and the serving scheduler
(``serving``).
"""
__all__ = ["native", "cell", "workloads", "recpot"]
