"""B200-native (sm_100a) RK3 step + multigrid pressure projection of the
anelastic/Boussinesq shear-layer solver, behind the reference's
mg_solver / rk_ss calling conventions (see include/anel.h)."""
from . import abi, grid  # noqa: F401

__version__ = "0.1.0"
