"""Coupled-cluster (T) drop-in: mirrors pyscfad.cc.ccsd_t on the B200 kernels."""
from . import ccsd_t  # noqa: F401
from .eris import ERIs  # noqa: F401
