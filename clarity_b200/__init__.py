"""clarity_b200 -- B200-native (sm_100a) implementation of Clarity's 3-D
FFT-convolution deconvolution path behind Clarity's C API.

The product is ``libclarity.so`` (C ABI, ``include/clarity.h``); this package
builds it (``clarity_b200.build``) and mirrors the C API in Python
(``clarity_b200.api``).  ``clarity_b200.synthetic`` generates the seeded test
volumes.
"""
from . import api  # noqa: F401
from .api import (ClarityError, convolve, maximum_likelihood_deconvolve,  # noqa: F401
                  blind_maximum_likelihood_deconvolve, wiener_deconvolve,
                  jansen_van_cittert_deconvolve, smoothed_jansen_van_cittert_deconvolve,
                  idivergence, register, unregister)

__version__ = "1.1.0"
