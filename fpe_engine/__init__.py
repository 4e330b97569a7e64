"""Import-compatible alias of the reference ``fpe_engine`` package.

``import fpe_engine as fpe`` keeps working for code written against the
reference (python/fpe_engine/__init__.py); the implementation is the
B200 engine in :mod:`fpe_option_b200`.
"""
from fpe_option_b200 import (  # noqa: F401
    Basis1DResult,
    Compute,
    FpeParams,
    GreeksResult,
    GridPointsResult,
    KnotsResult,
    PriceResult,
    is_available,
    price,
    __version__,
)
