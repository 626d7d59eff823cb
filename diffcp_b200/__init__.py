"""diffcp_b200: differentiable codimensional-cloth MPM (DiffCP's simulation.py
path) as hand-written sm_100a CUDA kernels behind a C ABI, batched over many
cloth instances on one B200.

Entry points:
  ClothBatch / BatchSim      batched rollouts and the autograd-enabled loss
  scene                      scene construction (reference normalisation, sheets)
  reference_api              drop-in module with the reference's names
"""
from . import native, scene  # noqa: F401

__all__ = ["native", "scene", "ClothBatch", "BatchSim"]


def __getattr__(name):
    if name in ("ClothBatch", "BatchSim"):
        from . import batch
        return getattr(batch, name)
    raise AttributeError(name)
