"""B200-native shoebox integration (the INTEGRATE stage of XPG): drop-in `integrate`, `estimate_sigmas`,
`IntegrationModel`, `IntegrationResult`, and XPG's inner kernel surface `make_kernels`, computed by hand-written
sm_100a CUDA kernels in libxpgi.so (C ABI: include/xpgi.h); `output` holds the stage's LP correction and its
`xpg_integrated.npz` / `INTEGRATE.HKL` writers."""
__version__ = "0.1.0"

from .device import keep_buffers  # noqa: F401
from .integrate import IntegrationResult, estimate_sigmas, integrate  # noqa: F401
from .kernels import make_kernels  # noqa: F401
from .plan import IntegrationModel  # noqa: F401
N_BOX = 5.0   # shoebox half-size in sigma units (xpg/integrate_kernels.py:15), read by the stage
