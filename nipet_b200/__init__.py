"""NIPET's reconstruction hot path for the Siemens mMR on B200 (sm_100a).

The CUDA kernels and their C ABI live in `libnipet_b200.so` (`csrc/`, built in-tree by
`nipet_b200.build`); the modules below mirror NIPET's Python surface on top of it:

* `petprj`, `mmrprj`: the projector extension (`tprj`, `fprj`, `bprj`, `osem`) and the
  `frwd_prj` / `back_prj` operators;
* `mmr_lmproc`, `mmrhist`: list-mode information, histogramming (with bootstrap) and
  randoms from the delayed fan sums;
* `mmraux`, `geometry`: sinogram gap conversion, scanner constants and look-up tables,
  and the reduced axial FOV (`reduce_rings`) the projectors also run in;
* `mmrnorm`: the normalisation sinogram from its components;
* `mmrrec`, `pipe`: OSEM on device-resident data, `osemone` and `mmrchain`;
* `mmrsct`: the voxel-driven scatter model and its estimate;
* `mmrsim`: sinogram simulation and reconstruction of simulated data;
* `batch`, `dynamic`, `diffprj`: batched bootstrap / dynamic-frame OSEM, the
  differentiable projector (autograd), and the batch-shape autotuner.

Submodules are imported on use; nothing here touches the GPU at import time.
"""
