"""LBM collision and streaming (reference physics/lbm.py)."""
from .. import kernels

collide_srt = kernels.collide_srt
collide_srt_variable_tau = kernels.collide_srt_variable_tau
collide_mrt = kernels.collide_mrt
stream = kernels.stream

__all__ = ["collide_srt", "collide_srt_variable_tau", "stream", "collide_mrt"]
