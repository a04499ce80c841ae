"""ctas_b200 -- B200-native parallel-beam filtered backprojection behind the
reconstruction interface of AustralianSynchrotron/ctas (class CTrec).

The compute path is the CUDA library ``libctas_fbp.so`` built from
``ctas_b200/csrc`` for sm_100a and reached through the C ABI of
``include/ctas_fbp.h``; this package holds the Python mirror of the
reference interface (``ct``), the phantom generator used for synthetic inputs
(``phantom``) and the build recipe (``build``).
"""
from .ct import CTrec, Contrast, CtasError, Filter, angle_table, padded_width, rec_cof  # noqa: F401

__version__ = "0.1.0"
