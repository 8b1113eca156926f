"""LNO (T) correction on B200 (mirrors pyscfad/lno)."""
from . import ccsd_t

__all__ = ["ccsd_t"]
