"""jax.scipy.linalg stand-in (dense LU, used by the reference's dense backend)."""

import scipy.linalg as _sla

from .._core import wrap


def lu_factor(a):
    lu, piv = _sla.lu_factor(a)
    return wrap(lu), wrap(piv)


def lu_solve(lu_piv, b):
    lu, piv = lu_piv
    return wrap(_sla.lu_solve((lu, piv), b))
