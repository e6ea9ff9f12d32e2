"""Quadrature of the pole density over one (omega, eta) data bin.

A pole-figure entry is the mean of a pole's Gaussian density over a bin. It is integrated with a tensor-product rule:
per direction, k panels of p-point Gauss-Legendre (p = 1: the midpoint rule). The rule for an operator is the one with
the fewest nodes per bin whose a-priori error bound, relative to the peak density and including the cut of the
Gaussian (exp(-pf_cutoff_sigma^2 / 2)), stays within a tolerance. Restates diffractom/operators/quadrature.py:1-222:

    bound per direction = c_p h^(2p) mu_(2p)(1 / sigma^2),  h = width / k,  c_p = (p!)^4 / ((2p + 1) ((2p)!)^3)

where mu_m(a) is the m-th moment of the symmetric Skellam distribution with parameter a (its even cumulants are a,
its odd ones 0), which bounds the m-th derivative of exp(a (cos t - 1)) along any omega or eta line.
"""
from __future__ import annotations

import warnings
from dataclasses import dataclass
from math import comb, factorial

import numpy as np

P_MAX = 8          # points per panel a rule may use
N_MAX = 64         # nodes per bin and direction a rule may use
DEFAULT_TOL = 0.05


def gauss_constant(p: int) -> float:
    """Error constant of the p-point Gauss-Legendre rule on one panel (1/24 for the midpoint rule)."""
    return factorial(p) ** 4 / ((2 * p + 1) * factorial(2 * p) ** 3)


def skellam_moment(m: int, a: float) -> float:
    """m-th moment (m even) of the symmetric Skellam distribution with parameter a: moments from cumulants
    (kappa_n = a for even n, 0 for odd n) by the recursion mu_n = sum_j C(n-1, j-1) kappa_j mu_(n-j)."""
    if m % 2:
        raise ValueError("m must be even")
    mu = [1.0]
    for n in range(1, m + 1):
        mu.append(sum(comb(n - 1, j - 1) * a * mu[n - j] for j in range(2, n + 1, 2)))
    return mu[m]


def direction_bound(p: int, k: int, width: float, sigma: float) -> float:
    h = abs(float(width)) / k
    return gauss_constant(p) * h ** (2 * p) * skellam_moment(2 * p, 1.0 / float(sigma) ** 2)


def nodes_weights(p: int, k: int):
    """Offsets in (0, 1) of a bin and weights (sum 1) of k panels of p-point Gauss-Legendre."""
    g, w = np.polynomial.legendre.leggauss(p)
    x = ((np.arange(k)[:, None] + 0.5 * (g[None, :] + 1.0)) / k).ravel()
    return x, np.tile(0.5 * w / k, k)


@dataclass(frozen=True)
class QuadratureRule:
    """k panels of p-point Gauss-Legendre per direction (omega, eta); p = 1 both ways: equal sub-bins."""
    p_omega: int = 1
    k_omega: int = 1
    p_eta: int = 1
    k_eta: int = 1

    def __post_init__(self):
        for v in (self.p_omega, self.k_omega, self.p_eta, self.k_eta):
            if int(v) != v or v < 1:
                raise ValueError(f"QuadratureRule needs positive integers, not {self}")

    @classmethod
    def midpoint(cls, n_omega: int = 1, n_eta: int = 1) -> "QuadratureRule":
        return cls(1, int(n_omega), 1, int(n_eta))

    @property
    def n_omega(self) -> int:
        return self.p_omega * self.k_omega

    @property
    def n_eta(self) -> int:
        return self.p_eta * self.k_eta

    @property
    def is_midpoint(self) -> bool:
        return self.p_omega == 1 and self.p_eta == 1

    def bound(self, d_omega: float, d_eta: float, sigma: float) -> float:
        return (direction_bound(self.p_omega, self.k_omega, d_omega, sigma)
                + direction_bound(self.p_eta, self.k_eta, d_eta, sigma))


def _best_per_count(width, sigma, p_max, n_max):
    """(n, bound, p, k) for n = 1 .. n_max: the smallest bound of any split n = p k."""
    rows = []
    for n in range(1, n_max + 1):
        cands = [(direction_bound(p, n // p, width, sigma), p, n // p) for p in range(1, min(p_max, n) + 1)
                 if n % p == 0]
        b, p, k = min(cands, key=lambda t: t[0])
        rows.append((n, b, p, k))
    return rows


def choose_rule(d_omega, d_eta, sigma, tol=DEFAULT_TOL, cut_share=0.0, p_max=P_MAX, n_max=N_MAX) -> QuadratureRule:
    """Fewest nodes per bin (then the smallest bound) with bound <= tol - cut_share."""
    budget = float(tol) - float(cut_share)
    if budget <= 0:
        raise ValueError(f"quadrature_tol = {tol:g} is not above the error of the Gaussian's cut ({cut_share:.2g})")
    om = _best_per_count(d_omega, sigma, p_max, n_max)
    et = _best_per_count(d_eta, sigma, p_max, n_max)
    best = None
    for nw, bw, pw, kw in om:
        for ne, be, pe, ke in et:
            if bw + be <= budget:
                key = (nw * ne, bw + be)
                if best is None or key < best[0]:
                    best = (key, QuadratureRule(pw, kw, pe, ke))
                break          # the first eta count that fits is the cheapest for this omega count
    if best is None:
        raise ValueError(f"no rule with at most {n_max} nodes per direction meets quadrature_tol = {tol:g} "
                         f"(sigma = {np.degrees(sigma):.3g} deg)")
    return best[1]


def cut_share(pf_cutoff_sigma) -> float:
    """exp(-PF_CUT): the largest error of a PF entry, relative to the peak, from the cut of the Gaussian."""
    return float(np.exp(-pf_cut_value(pf_cutoff_sigma)))


def pf_cut_value(pf_cutoff_sigma) -> float:
    """The exponent at which the Gaussian is cut: pf_cutoff_sigma^2 / 2 (6 when None, the historic threshold)."""
    return 6.0 if pf_cutoff_sigma is None else float(pf_cutoff_sigma) ** 2 / 2


@dataclass
class QuadratureSetup:
    rule: QuadratureRule
    bound: float
    omega_nodes: np.ndarray      # (N_Omega * S,) the nodes, bin by bin
    eta_nodes: np.ndarray        # (N_eta * S_eta,)
    weights: np.ndarray | None   # (S * S_eta,) float32 product weights; None for the midpoint rule (averaged)


def setup_quadrature(angle_range, n_omega, eta_range, n_eta, cfg, quadrature, tol, sigma_min, pf_cutoff_sigma):
    """The rule and its nodes for an operator (angle ranges in radians), as diffractom's setup_quadrature
    (quadrature.py:168-222): "auto" picks the rule, "midpoint" takes cfg's N_Omega_subdivisions / N_eta_subdivisions,
    a QuadratureRule is used as given. Equal sub-bins keep the linspace node expression of earlier versions."""
    a0, a1 = float(angle_range[0]), float(angle_range[1])
    e0, e1 = float(eta_range[0]), float(eta_range[1])
    delta = (a1 - a0) / n_omega
    eta_delta = (e1 - e0) / n_eta
    share = cut_share(pf_cutoff_sigma)
    given = [k for k in ("N_Omega_subdivisions", "N_eta_subdivisions") if k in cfg]
    if isinstance(quadrature, QuadratureRule):
        rule = quadrature
    elif quadrature == "midpoint":
        rule = QuadratureRule.midpoint(cfg.get("N_Omega_subdivisions", 1), cfg.get("N_eta_subdivisions", 1))
    elif quadrature == "auto":
        rule = choose_rule(delta, eta_delta, sigma_min, tol, share)
        if given and any(int(cfg[k]) != 1 for k in given):
            warnings.warn(f"{' and '.join(given)} are used only with quadrature='midpoint'", stacklevel=3)
    else:
        raise ValueError(f"quadrature must be 'auto', 'midpoint' or a QuadratureRule, not {quadrature!r}")
    S, Se = rule.n_omega, rule.n_eta
    if rule.p_omega == 1:
        om = np.linspace(a0, a1, n_omega * S, endpoint=False) + delta / S / 2
    else:
        x, _ = nodes_weights(rule.p_omega, rule.k_omega)
        om = (a0 + (np.arange(n_omega)[:, None] + x[None, :]) * delta).ravel()
    if rule.p_eta == 1:
        et = np.linspace(e0, e1, n_eta * Se, endpoint=False) + eta_delta / Se / 2
    else:
        x, _ = nodes_weights(rule.p_eta, rule.k_eta)
        et = (e0 + (np.arange(n_eta)[:, None] + x[None, :]) * eta_delta).ravel()
    if rule.is_midpoint:
        w = None
    else:
        _, ww = nodes_weights(rule.p_omega, rule.k_omega)
        _, we = nodes_weights(rule.p_eta, rule.k_eta)
        w = np.ascontiguousarray((ww[:, None] * we[None, :]).ravel(), dtype=np.float32)
    return QuadratureSetup(rule, rule.bound(delta, eta_delta, sigma_min) + share, om, et, w)
