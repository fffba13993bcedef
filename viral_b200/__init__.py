"""B200-native viscous Kurganov-Tadmor hydro step (the hot path of
rjfries/VIRAL) behind the C ABI in include/vh.h."""
from .hydro import HBARC, A_QGP, Config, Hydro, eos_table_synthetic, profile_glauber, profile_gubser  # noqa: F401
from . import _abi as abi  # noqa: F401
from . import configs  # noqa: F401
