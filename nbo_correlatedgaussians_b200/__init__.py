"""B200 engine for the energy-and-gradient hot path of NECG
(MauricioCafiero/NBO_CorrelatedGaussians): explicitly correlated Gaussians,
non-Born-Oppenheimer, FP64.

Drop-in modules with the reference's names and signatures:
  read_input.read_input, matel.matel, gradel.gradel, make_grad.make_grad,
  outprod.outprod, utils.f0 / df0 / vech, shared (module state)
Engine-level API: engine.Engine, autograd.EnergyFn, batch.BatchEngine,
serve.Server.  All arithmetic runs in libnecg_b200.so (CUDA, sm_100a).
"""
from .problem import Problem, read_oldquit, write_oldquit  # noqa: F401

__all__ = ["Problem", "read_oldquit", "write_oldquit"]
