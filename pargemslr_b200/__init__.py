"""pargemslr_b200: a B200-native solve phase for ParGeMSLR's GeMSLR-FGMRES.

The reference ParGeMSLR (Hitenze/pargemslr) builds a multilevel Schur
low-rank preconditioner on the host; this package runs the SOLVE phase on one
GPU with hand-written sm_100a kernels behind the C ABI of ``include/pgx.h``.
"""
from . import params  # noqa: F401
from .structures import GemslrStructures, LevelStructures, from_dump  # noqa: F401

__all__ = ["params", "GemslrStructures", "LevelStructures", "from_dump", "GemslrHandle"]


def __getattr__(name):
    if name == "GemslrHandle":
        from .handle import GemslrHandle
        return GemslrHandle
    raise AttributeError(name)
