from .lippmann_schwinger import (  # noqa: F401
    CONVERGED, MAXITER, NONFINITE, PRECISIONS, STALLED, RULE_CUDA, RULE_JAX, Solver, SolveResult, c_eff,
    lippmann_schwinger, lippmann_schwinger_cuda, lippmann_schwinger_jax)
from .gradient import EffectiveStiffness, c_eff_autograd  # noqa: F401,E402
from .batch import c_eff_batch  # noqa: F401,E402
from .distributed import assign_lpt, c_eff_batch_sharded  # noqa: F401,E402
