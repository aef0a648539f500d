"""B200 (sm_100a) hot path of block-DDA: doubled-grid FFT MVP + block Krylov solvers.

The reference's own module paths (``mvp_fft.mvp_fft``, ``bl_krylov.bl_krylov``,
``bl_dda.scatterer``) are provided as siblings of this package; put the
``block-dda_py_b200`` folder on ``sys.path`` in place of the reference's root.
"""
from . import _lib  # noqa: F401

__version__ = "0.1.0"
