"""B200 (sm_100a) implementation of the MuhRec reconstruction hot path.

``modules`` holds the reference-compatible modules (FullLogNorm, ProjectionFilterSingle,
MultiProjectionBPparallel, FDKbp_single), ``pipeline`` device-resident chains of them,
``phantom`` seeded synthetic inputs; the kernels live in ``libmrcuda.so`` (C ABI in
``include/mrcuda.h``), built by ``imagingsuite_b200.build``.
"""
__version__ = "0.1.0"
