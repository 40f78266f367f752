"""tensorsvm_b200: B200-native TensorSVM training path (kernel factor + SMW interior point).

The compute lives in the CUDA library libtensorsvm_b200.so (C ABI: include/tensorsvm.h);
``train`` below drives it from Python for users and tests, the ``tensorsvm-train`` CLI drives
it from C++ with the reference's command line.
"""
from . import _lib
from .api import Model, factor, ipm, bias, train, write_model, read_libsvm

__all__ = ["Model", "factor", "ipm", "bias", "train", "write_model", "read_libsvm", "_lib"]
