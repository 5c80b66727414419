"""magic_b200 — B200-native pseudo-spectral nonlinear stage for torch-magic.

Hand-written sm_100a CUDA behind a C ABI (include/magic_b200.h,
libmagic_b200.so), driven from Python through ctypes on torch CUDA tensors.

* ``magic_b200.Plan``        one (l_max, minc) resolution on one GPU
* ``magic_b200.sht``         drop-in for ``magic_torch.sht`` (same signatures)
* ``magic_b200.get_nl``      drop-in for get_nl / get_nl_anel / courant_check
* ``Plan.nl_bouss``          the fused radial-loop nonlinear stage
"""

from ._lib import MagicError  # noqa: F401
from .config import configure, configure_from_reference  # noqa: F401
from .plan import Plan  # noqa: F401

__version__ = "0.1.0"
