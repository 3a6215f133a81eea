"""magtense_b200: B200-native micromagnetic hot path of MagTense.

The Landau-Lifshitz right-hand side (dense prism demag tensor, exchange,
anisotropy, Zeeman), the analytical prism-tensor assembly and the RKSUITE-90
'M' adaptive integration run in hand-written sm_100a kernels behind the C ABI
of ``libmagtense_b200.so`` (``include/magtense_b200.h``).  ``MicromagProblem``
mirrors ``magtense.micromag.MicromagProblem``.
"""
from ._lib import LIB_PATH, MTError, build, lib  # noqa: F401


def __getattr__(name):
    # torch-dependent modules are imported lazily so that the C ABI can be
    # inspected on machines without a GPU
    if name in ("MicromagProblem", "load_demag_tensor", "save_demag_tensor"):
        from . import micromag
        return getattr(micromag, name)
    if name in ("Solver", "BatchSolver", "grid_points", "integrate_ragged", "shard_rows", "link_shards_local",
                "integrate_shards_local"):
        from . import solver
        return getattr(solver, name)
    if name == "dataset":
        import importlib
        return importlib.import_module(".dataset", __name__)
    if name in ("TrajectoryProblem", "mean_m_trajectory", "LLTrajectory"):
        from . import adjoint
        return getattr(adjoint, name)
    raise AttributeError(name)
