"""fastwarp_b200 -- the registration hot path of WyssCenter/fastwarp on B200 (sm_100a) GPUs.

The engine is the CUDA library ``libfastwarp_cuda.so`` behind the C ABI in
``include/fastwarp_cuda.h``; this package is its Python host mirror:

  - `CudaBackend` -- the operations of the reference's `Backend` trait (SyN loop);
  - `CudaLinearEngine` / `MiLevel` -- `LinearEngine` / `LinearMetric` (sampled Mattes MI);
  - `run_syn` -- the SyN stage, one CUDA graph launch per pyramid level;
  - `run_syn_batch` -- many subjects to one template in lockstep (persistent batched kernels);
  - `serve` -- the continuous-batching request server (several registrations in flight).
"""
from ._native import FastwarpError, build, lib
from .backend import (CudaBackend, CudaLinearEngine, Field, Image, MiLevel, binning_from_ranges,
                      grid_shape, linear_transform, make_affine, make_grid, shrink_factors,
                      shrink_grid)
from .syn import (BatchResult, SynRecipe, SynResult, level_grid, run_syn, run_syn_batch,
                  run_syn_device, run_syn_from, syn_step)

__all__ = [
    "FastwarpError", "build", "lib", "CudaBackend", "CudaLinearEngine", "Field", "Image",
    "MiLevel", "binning_from_ranges", "grid_shape", "linear_transform", "make_affine",
    "make_grid", "shrink_factors", "shrink_grid", "SynRecipe", "SynResult", "level_grid",
    "run_syn", "run_syn_batch", "run_syn_device", "run_syn_from", "syn_step", "BatchResult",
]
