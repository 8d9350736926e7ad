"""B200-native LenseFlow engine with the interface of zaneblood1/CMBLensing.py's lensing path."""
from .constants import (FORWARD_LENSE, INVERSE_LENSE, NSIDE_DEFAULT, PIX_WIDTH_DEFAULT, THETA_PIX_DEFAULT, Basis,
                        Parametrization, Polarity)
from .fields import (FlatS0, FlatS02, FlatS2, dot, eb2qu, fourier, fourier_weights_default, get_fourier_weights,
                     map, qu2eb)

__version__ = "0.1.0"


_LAZY_MODULES = ("engine", "simulate", "build")


def __getattr__(name):
    # torch-dependent modules load lazily so the containers import without CUDA
    import importlib
    if name == "lense_flow":
        return importlib.import_module(".lense_flow", __name__).lense_flow
    if name in _LAZY_MODULES:
        return importlib.import_module("." + name, __name__)
    raise AttributeError(name)
