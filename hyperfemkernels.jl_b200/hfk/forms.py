"""Weak forms the engine recognises (the laws the kernels implement).

In the reference the host captures the user's Gridap closures into an expression tree
(``capture``, HyperFEMKernels ``src/tree.jl:74-98``) and generates a pointwise function. The GPU
cannot call Julia code, so the host recognises the law from the tree's structure and passes its
parameters to the kernels. This module is that recognised form in Python: a residual form and a
Jacobian form of the same law, parameters and quadrature degree.

* ``svk_*``: St Venant-Kirchhoff, P(F) = F S, S = lambda tr(E) I + 2 mu E, E = (F'F - I)/2
  (``test/common.jl:1-8``, ``README.md:61-67``), with an optional constant body force
  (``- v . body``, ``test/solvers/test_pmultigrid.jl:21-22``);
* ``linear_elastic_*``: sigma = lambda tr(G) I + mu (G + G') (``test/solvers/test_pmultigrid.jl:9``).
"""
from __future__ import annotations

import dataclasses

from . import _lib


@dataclasses.dataclass(frozen=True)
class Form:
    """A recognised integrand on a volume measure of quadrature ``degree``."""

    law: int
    lam: float
    mu: float
    degree: int
    body: tuple = (0.0, 0.0, 0.0)
    kind: str = "res"  # "res" or "jac"

    def params(self):
        return [float(self.lam), float(self.mu)] + [float(b) for b in self.body]

    def same_law(self, other: "Form") -> bool:
        return (self.law, self.lam, self.mu, self.degree) == (other.law, other.lam, other.mu, other.degree)


def svk_residual(lam=2.0, mu=1.0, degree=4, body=(0.0, 0.0, 0.0)) -> Form:
    return Form(_lib.LAW_SVK, lam, mu, degree, tuple(body), "res")


def svk_jacobian(lam=2.0, mu=1.0, degree=4) -> Form:
    return Form(_lib.LAW_SVK, lam, mu, degree, (0.0, 0.0, 0.0), "jac")


def linear_elastic_residual(lam=2.0, mu=1.0, degree=4, body=(0.0, 0.0, 0.0)) -> Form:
    return Form(_lib.LAW_LINEAR_ELASTIC, lam, mu, degree, tuple(body), "res")


def linear_elastic_jacobian(lam=2.0, mu=1.0, degree=4) -> Form:
    return Form(_lib.LAW_LINEAR_ELASTIC, lam, mu, degree, (0.0, 0.0, 0.0), "jac")
