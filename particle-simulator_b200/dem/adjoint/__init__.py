from .direct_adjoint import DirectTrajectory, mean_squared_z_displacement, pair_softplus

__all__ = ["DirectTrajectory", "mean_squared_z_displacement", "pair_softplus"]
