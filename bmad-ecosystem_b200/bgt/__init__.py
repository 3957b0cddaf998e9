"""bgt -- B200-native FP64 multi-particle tracker for Bmad bmad_standard lattices.

Host-side package: lattice model and bookkeeping (:mod:`bgt.lattice`),
synthetic rings (:mod:`bgt.rings`), optics (:mod:`bgt.optics`), the tracker
handle over the CUDA library (:mod:`bgt.track`), dynamic-aperture scans
(:mod:`bgt.da`), the survival classifier (:mod:`bgt.mlp`) and the launch-tile
autotuner (:mod:`bgt.autotune`).  The compute path is libbgt.so (sm_100a).
"""
from . import lattice, optics, rings  # noqa: F401
