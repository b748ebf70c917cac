"""LBM collision and streaming (reference physics/lbm.py)."""
from .. import kernels
from .._native import WaamError

collide_srt = kernels.collide_srt
collide_mrt = kernels.collide_mrt
stream = kernels.stream


def collide_srt_variable_tau(*args, **kwargs):
    """kernels.py:2888-2965 -- material-table path, not built in this backend."""
    raise WaamError("collide_srt_variable_tau (material-table path) is not supported; "
                    "use a constants-only material")


__all__ = ["collide_srt", "collide_srt_variable_tau", "stream", "collide_mrt"]
