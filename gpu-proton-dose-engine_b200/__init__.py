"""B200-native separable proton pencil-beam dose engine.

Drop-in for the reference's per-layer exact separable engine
(``engines.torch_separable(per_layer=True)``, engines.py:208-283) behind the same
``PBProblem`` / ``DoseGrid`` / ``SpotLattice`` API (model.py:27-187), computed by
hand-written sm_100a CUDA in ``libpbdose_b200.so`` through a C ABI
(``include/pbdose_b200.h``).  There is no CPU path: calls that need the device raise
when the library or a CUDA device is missing.

The directory name is not a Python identifier; import it with
``importlib.import_module("gpu-proton-dose-engine_b200")``.  After that, the alias
``pbdose_b200`` (and ``pbdose_b200.<submodule>``) refers to the same modules.

Modules
  model      DoseGrid, SpotLattice, PBProblem and the field builders
  physics    device depth-LUT builder (FP64) and range-table lookups
  engines    torch_separable, the autograd function, the fused loss gradient
  robust     batched fields x scenarios in one persistent launch, CUDA graphs
  optimize   on-device plan optimisation (projected Adam, robust mean / min-max), CUDA graphs
  gamma      gamma index (the reference's gamma.py) in one device call, float64 semantics
  hetero     water-equivalent depth ray trace and the dose in heterogeneous media
  tuning     measured choice of the work-item sizes, cached per geometry
  distributed  depth-slab and job sharding over torch.distributed (one GPU per rank)
  workloads  synthetic workloads of the benchmark shapes (host, NumPy)
"""
import sys as _sys

from . import workloads, _lib, physics, model, engines, robust, tuning, distributed, optimize, gamma, hetero  # noqa: F401,E501

__version__ = "0.1.0"

_sys.modules.setdefault("pbdose_b200", _sys.modules[__name__])
for _name in ("workloads", "_lib", "physics", "model", "engines", "robust", "tuning",
              "distributed", "optimize", "gamma", "hetero"):
    _sys.modules.setdefault("pbdose_b200." + _name, _sys.modules[__name__ + "." + _name])
