"""B200-native elastic spectral-element forward/adjoint time loop.

Drop-in for the hot path of SpecFWAT's ``xfwat_fwd_measure_adj``: the C ABI
in ``include/sem_b200.h`` (``libsem_b200.so``), and this Python mirror of
the reference's per-event driver (:mod:`specfwat_b200.solver`).  Kernel
smoothing on the device is :mod:`specfwat_b200.postproc`; the serving loop
:mod:`specfwat_b200.serving`.  The mesh and model generator for the
standard workloads is :mod:`specfwat_b200.database`.
"""
__version__ = "0.1.0"
