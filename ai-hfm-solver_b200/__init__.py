"""ai-hfm-solver_b200: B200-native stencil operators and geometric multigrid for the
AI4CFD (bc1chen/AI-HFM-Solver) hot path.

Import name: ``ai_hfm_solver_b200`` (the directory name has hyphens; ``__graft_entry__``
provides ``load_package()`` which registers it).  All compute runs in ``libhfm.so``
(hand-written sm_100a kernels behind a C ABI, ``include/hfm.h``); torch tensors are the
I/O container only.
"""
from . import _lib  # noqa: F401
from . import weights  # noqa: F401
from . import problems  # noqa: F401

__all__ = ["_lib", "weights", "problems", "ops", "multigrid"]


def __getattr__(name):
    # ops / multigrid import torch; keep the package importable for the build step.
    if name in ("ops", "multigrid", "serving", "precision", "tomography", "ns", "kolmogorov",
                "slab"):
        import importlib
        return importlib.import_module("." + name, __name__)
    raise AttributeError(name)
