"""B200 (sm_100a) implementation of ATJUP's time-step hot path.

The CUDA kernels and the C ABI live in ``atjup_b200/csrc`` and are built in-tree into
``atjup_b200/libatjup_gpu.so`` (``python -m atjup_b200.build``). ``atjup_b200.gpu`` binds that
library; ``atjup_b200.params`` resolves the reference's environment knobs on the host.
"""
__all__ = ["params"]
