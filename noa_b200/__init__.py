"""noa_b200: B200-native (sm_100a) Fourier central-slice extraction and insertion.

Drop-in for noa's ``noa::xform`` central-slice functions (noa/xform/FourierProject.hpp); see
``noa_b200.fourier_project`` for the host API and ``include/noa_b200/fourier_project.h`` for the C ABI.

Modules:
  fourier_project  the four central-slice functions, the scatter-form insertion, the gridding correction
  batch            many extractions in one persistent launch (CUDA graph, autotuned); pair copies
  serve            serving loop: HBM-budget admission, continuous batching, latency accounting
  reconstruct      spectrum normalization + remap + centering, cuFFT c2r, gridding correction
  shard            multi-GPU slice sharding and grid all-reduce (one process per GPU)
  mrc              MRC2014 files
  synthetic        seeded synthetic volumes, slices and orientations
  workloads        the batched and served workloads (python -m noa_b200.workloads ...)
  build            builds the CUDA library in tree (python -m noa_b200.build)
"""
