"""fcwt_b200 — B200-native (sm_100a) fast continuous wavelet transform.

Drop-in for the transform path of fastlib/fCWT: ``import fcwt_b200 as fcwt``
gives the reference module's names (Morlet, Scales, FCWT with cwt/ccwt,
create_FFT_optimization_plan, the FCWT_* scale types and the ``cwt``
boilerplate). The transform runs in hand-written CUDA kernels behind the C ABI
of lib/libfcwt_b200.so; there is no CPU fallback.
"""
from ._lib import (FcwtError, FCWT_OUT_BF16, FCWT_OUT_C64, FCWT_OUT_DB, FCWT_OUT_F16,  # noqa: F401
                   FCWT_OUT_POWER, LIB_PATH)
from .api import (DOG, FCWT, FCWT_LINFREQS, FCWT_LINSCALES, FCWT_LOGSCALES, BatchPlan, Morlet, Paul, Plan,  # noqa: F401
                  Scales, Wavelet, cwt, cwt_device, mother_host, row_truncation, synchronize)

__all__ = ["Morlet", "Paul", "DOG", "Scales", "FCWT", "Wavelet", "FCWT_LINSCALES", "FCWT_LOGSCALES", "FCWT_LINFREQS", "cwt",
           "cwt_device", "Plan", "BatchPlan", "synchronize", "row_truncation", "mother_host", "FcwtError",
           "morlet_cwt", "morlet_power_cwt", "LearnableMorletCWT"]


def __getattr__(name):
    if name == "StreamingCWT":
        from .streaming import StreamingCWT

        return StreamingCWT
    # the differentiable operator needs torch; import it on first use
    if name in ("morlet_cwt", "morlet_power_cwt", "LearnableMorletCWT", "MorletCWTFunction", "MorletPowerFunction"):
        from . import autograd

        return getattr(autograd, name)
    raise AttributeError(name)
