"""mcsart_b200 - B200-native McSART engine (motion-compensated SART CBCT).

The compute lives in ``lib/libmcsart.so`` (hand-written CUDA for sm_100a behind
the C ABI of include/mcsart.h).  This package is the host-side mirror of the
reference's interface:

  * ``Context``: one method per reference launcher (``host_projection``,
    ``host_backprojection``, ``host_deform``, ... , ``host_AUMISART``) plus the
    device-resident driver ``aumisart_device``;
  * ``gateway``: the three MATLAB gateways (``entry_AUMISART``,
    ``mex_backprojection``, ``mex_diff``) with their struct parsing;
  * ``synthetic``: seeded phantoms, geometry and 5DCT motion for the benchmarks.
"""
from ._lib import (BF16, ERR_CUDA, ERR_INVALID_ARGUMENT, ERR_NO_DEVICE, ERR_OUT_OF_MEMORY, F16,
                   F32, INTERP_EXACT, INTERP_TEXTURE, LIB_PATH, McsartError, Options)
from .engine import Context, default_options, projection_noalloc

__version__ = "1.0.0"
__all__ = ["Context", "McsartError", "Options", "default_options", "projection_noalloc", "LIB_PATH", "F32", "BF16",
           "F16", "INTERP_TEXTURE", "INTERP_EXACT", "ERR_CUDA", "ERR_INVALID_ARGUMENT",
           "ERR_NO_DEVICE", "ERR_OUT_OF_MEMORY"]
