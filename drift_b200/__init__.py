"""drift_b200 - B200-native parallel-tempering engine behind DRiFT's PT entry point.

    from drift_b200.gpu import gpu_available, parallel_tempering_gpu   # drop-in for drift.gpu
    from drift_b200.ising import IsingModel, SparseIsingModel

The compute path is libdrift_pt.so (hand-written sm_100a CUDA behind the C ABI in
include/drift_pt.h), built in-tree by ``python -m drift_b200.build``.
"""

__version__ = "0.1.0"
