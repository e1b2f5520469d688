"""B200 execution backend for DogQC relational plans.

Front end (same API as the reference): ``relational``, ``scalar``, ``types``.
Backend: ``backend.Backend`` (drop-in for ``CudaCompiler``), ``engine.Engine``
(C-ABI handle on the CUDA engine in ``libdogqc_b200.so``), ``lowering`` (plan
tree -> pipeline IR).  Workloads: ``workloads``.
"""
__all__ = ["relational", "scalar", "types", "backend", "engine", "lowering", "workloads", "database"]
