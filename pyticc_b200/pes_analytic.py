"""Analytic atom-diatom PES in the Legendre-expansion form, evaluated on the host or on the GPU.

The reference takes the interaction PES as a user callable and evaluates it on the host on
the tensor grid of ``src/pyticc/pes/adiabatic.py:109-137`` (``get_Vgrid_atom_diatom``: R x r x
theta, meshgrid "ij" order).  A PES written declaratively as

    V(R, r, theta) = sum_t P_lam_t(cos theta) * f_t(R) * g_t(r - re),
    f_t(R) = sum of radial primitives,   g_t(d) = sum_q c_tq d^q,

is a ``LegendrePES``: it is a ``PESWrapper`` (its ``interaction`` evaluates the same sum with
NumPy, so it can stand wherever a user PES does) and ``prepare_potential`` fills its grid
directly in device memory with ``ticc_pes_legendre_grid`` when a GPU is present, so the
PotentialGrid of a long radial grid needs neither a host evaluation nor a host-to-device copy.

Radial primitives (``Primitive(kind, a, b, c)``):
    "power"  a R^-b            "exp"  a exp(-b (R - c))
    "gauss"  a exp(-((R - c)/b)^2)       "lj"   a ((b/R)^12 - 2 (b/R)^6)
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch
from loguru import logger

from . import _native as nat
from .pes import PESWrapper

KINDS = {"power": 0, "exp": 1, "gauss": 2, "lj": 3}
MAX_TERMS, MAX_PRIM, MAX_POLY, MAX_LAM = 16, 4, 4, 32


@dataclass(frozen=True)
class Primitive:
    kind: str
    a: float
    b: float
    c: float = 0.0

    def __post_init__(self):
        if self.kind not in KINDS:
            message = f"unknown radial primitive {self.kind!r}; expected one of {sorted(KINDS)}"
            logger.error(message)
            raise ValueError(message)

    def __call__(self, R: np.ndarray) -> np.ndarray:
        if self.kind == "power":
            return self.a * R ** (-self.b)
        if self.kind == "exp":
            return self.a * np.exp(-self.b * (R - self.c))
        if self.kind == "gauss":
            z = (R - self.c) / self.b
            return self.a * np.exp(-(z * z))
        s = self.b / R
        s6 = (s * s) * (s * s) * (s * s)
        return self.a * (s6 * s6 - 2.0 * s6)


@dataclass(frozen=True)
class LegendreTerm:
    """P_lam(cos theta) * sum(radial)(R) * sum_q poly[q] (r - re)^q."""

    lam: int
    radial: tuple[Primitive, ...]
    poly: tuple[float, ...] = (1.0,)


def _legendre(lmax: int, x: np.ndarray) -> list[np.ndarray]:
    """P_0 .. P_lmax by the three-term recurrence (the kernel's order of operations)."""
    P = [np.ones_like(x)]
    if lmax >= 1:
        P.append(x.copy())
    for l in range(1, lmax):
        P.append(((2 * l + 1) * x * P[l] - l * P[l - 1]) / (l + 1))
    return P


@dataclass(frozen=True)
class LegendrePES(PESWrapper):
    """An atom-diatom interaction PES in the Legendre-expansion form (see the module text)."""

    terms: tuple[LegendreTerm, ...] = ()
    re: float = 0.0

    @classmethod
    def build(cls, terms, re: float = 0.0) -> "LegendrePES":
        terms = tuple(terms)
        if not 1 <= len(terms) <= MAX_TERMS:
            message = f"a LegendrePES takes 1 to {MAX_TERMS} terms, got {len(terms)}"
            logger.error(message)
            raise ValueError(message)
        for t in terms:
            if not (0 <= int(t.lam) <= MAX_LAM and len(t.radial) <= MAX_PRIM and 1 <= len(t.poly) <= MAX_POLY):
                message = f"term {t} is outside the supported form (lam <= {MAX_LAM}, at most {MAX_PRIM} primitives and {MAX_POLY} coefficients)"
                logger.error(message)
                raise ValueError(message)
        holder: dict = {}

        def interaction(R, coordinates):
            return holder["pes"].evaluate(R, coordinates)

        pes = cls(interaction=interaction, terms=terms, re=float(re))
        holder["pes"] = pes
        return pes

    # ---- host evaluation (the PESWrapper contract) ----------------------------------------
    def evaluate(self, R, coordinates) -> np.ndarray:
        """V at one radial point R for coordinates (r, theta) of shape (2, n_grid)."""
        r, theta = np.asarray(coordinates, dtype=np.float64)
        x = np.cos(theta)
        d = r - self.re
        P = _legendre(max(t.lam for t in self.terms), x)
        RR = float(R)
        v = np.zeros_like(x)
        for t in self.terms:
            f = 0.0
            for p in t.radial:
                f = f + float(p(np.float64(RR)))
            g = np.zeros_like(d)
            for c in reversed(t.poly):
                g = g * d + c
            v = v + P[t.lam] * f * g
        return v

    # ---- device evaluation ---------------------------------------------------------------
    def _tables(self):
        n = len(self.terms)
        lam = (ctypes.c_int * n)(*[int(t.lam) for t in self.terms])
        n_prim = (ctypes.c_int * n)(*[len(t.radial) for t in self.terms])
        n_poly = (ctypes.c_int * n)(*[len(t.poly) for t in self.terms])
        kinds = (ctypes.c_int * (n * MAX_PRIM))()
        params = (ctypes.c_double * (n * MAX_PRIM * 3))()
        poly = (ctypes.c_double * (n * MAX_POLY))()
        for i, t in enumerate(self.terms):
            for j, p in enumerate(t.radial):
                kinds[i * MAX_PRIM + j] = KINDS[p.kind]
                params[(i * MAX_PRIM + j) * 3 + 0] = p.a
                params[(i * MAX_PRIM + j) * 3 + 1] = p.b
                params[(i * MAX_PRIM + j) * 3 + 2] = p.c
            for q, c in enumerate(t.poly):
                poly[i * MAX_POLY + q] = c
        return n, lam, n_prim, kinds, params, n_poly, poly

    def grid_device(self, R, r, cos_theta, device) -> torch.Tensor:
        """V on the (R, r, theta) tensor grid as a device tensor of shape (n_R, n_r * n_theta)."""
        dev = torch.device(device)
        lib = nat.load_library()
        Rt = torch.as_tensor(np.ascontiguousarray(R, dtype=np.float64), device=dev)
        rt = torch.as_tensor(np.ascontiguousarray(r, dtype=np.float64), device=dev)
        xt = torch.as_tensor(np.ascontiguousarray(cos_theta, dtype=np.float64), device=dev)
        V = torch.empty((Rt.numel(), rt.numel() * xt.numel()), dtype=torch.float64, device=dev)
        n, lam, n_prim, kinds, params, n_poly, poly = self._tables()
        nat.check(
            lib.ticc_pes_legendre_grid(nat.ptr(Rt), Rt.numel(), nat.ptr(rt), rt.numel(), nat.ptr(xt), xt.numel(), n, lam, n_prim, kinds, params, n_poly, poly, self.re, nat.ptr(V),
                                       nat.stream_handle(dev)),
            "ticc_pes_legendre_grid",
        )
        return V


# ---- the benchmark systems' analytic surfaces in this form ----------------------------------------
def lj_aniso_legendre(eps: float, Rm: float, a1: float, a2: float, c1: float = 0.0, c2: float = 0.0, re: float = 1.4) -> LegendrePES:
    """eps [(Rm/R)^12 - 2 (Rm/R)^6] (1 + a1 (1 + c1 (r - re)) P1 + a2 (1 + c2 (r - re)) P2), eps in hartree."""
    lj = (Primitive("lj", eps, Rm),)
    return LegendrePES.build([LegendreTerm(0, lj), LegendreTerm(1, lj, (a1, a1 * c1)), LegendreTerm(2, lj, (a2, a2 * c2))], re=re)


def capture_legendre(C6: float, wall: float, g: tuple[float, float, float]) -> LegendrePES:
    """-C6/R^6 (1 + 0.1 P2) + wall exp(-((R - 7)/1.5)^2) (g0 + g1 P1 + g2 P2), wall in hartree."""
    w = [Primitive("gauss", wall * gk, 1.5, 7.0) for gk in g]
    return LegendrePES.build(
        [LegendreTerm(0, (Primitive("power", -C6, 6.0), w[0])), LegendreTerm(1, (w[1],)), LegendreTerm(2, (Primitive("power", -0.1 * C6, 6.0), w[2]))]
    )
