"""Coupling slots of pNED's local Hamiltonian.

The reference keeps its couplings in module variables
(S_one_half/Hybrid_TPS_params.f90:17-26) that ``set_xlocal_Ham`` turns into 3x3
exchange matrices per bond type (:1441-1465).  This module names those 19
slots and maps the physical parameters of the measured workloads onto them.

Slot meaning for the nearest-neighbour types (J1x/J1y/J1z of the reference):

* ``K1``  -- S^z S^z coefficient on z-bonds (type 3), i.e. J + K,
* ``K1p`` -- S^x S^x on x-bonds and S^y S^y on y-bonds (J + K),
* ``J1``  -- S^x S^x, S^y S^y on z-bonds; ``J1p``/``J1pp`` the other
  Heisenberg components on x/y bonds,
* ``I11`` -- Gamma on the off-diagonal pair of z-bonds (S^x S^y + S^y S^x),
* ``I11p`` -- Gamma on x-bonds (S^y S^z + S^z S^y) and y-bonds (S^z S^x + S^x S^z),
* ``I12``, ``I12p``, ``I12pp`` -- Gamma' slots.
"""
from __future__ import annotations

import math

import numpy as np

SLOTS = ("J1", "K1", "I11", "I12", "J1p", "K1p", "J1pp", "K1pp", "I11p", "I12p",
         "I11pp", "I12pp", "J2", "K2", "I21", "I22", "J3", "K3", "ratio_l")
NSLOT = len(SLOTS)


def slots(**kw) -> np.ndarray:
    """Slot vector with the reference's defaults (all zero, ratio_l = 1)."""
    out = np.zeros(NSLOT)
    out[SLOTS.index("ratio_l")] = 1.0
    for k, v in kw.items():
        out[SLOTS.index(k)] = v
    return out


def kitaev_heisenberg(J: float, K: float, gamma: float = 0.0, gamma_p: float = 0.0) -> np.ndarray:
    """H = sum_<ij>_g [ J S_i.S_j + K S_i^g S_j^g + Gamma (S^a S^b + S^b S^a) + Gamma' ... ].

    The Kitaev slot of each bond type carries the full J + K coefficient, as
    MODEL 20 does (params.f90:171).
    """
    return slots(J1=J, K1=J + K, J1p=J, K1p=J + K, J1pp=J, K1pp=J + K,
                 I11=gamma, I11p=gamma, I11pp=gamma, I12=gamma_p, I12p=gamma_p, I12pp=gamma_p)


def model20(param_deg: float) -> np.ndarray:
    """MODEL 20 of set_lattice (params.f90:167-181): J = cos a, K-slot = cos a + 2 sin a."""
    a = 4.0 * math.atan(1.0) / 180.0 * param_deg
    J1 = math.cos(a)
    K1 = math.cos(a) + 2.0 * math.sin(a)
    return slots(J1=J1, K1=K1, J1p=J1, K1p=K1, J1pp=J1, K1pp=K1)


def model0(alp: float) -> np.ndarray:
    """MODEL 0 of set_lattice (params.f90:152-166): J = 1 - a, K-slot = 1 - 3a."""
    return slots(J1=1 - alp, K1=1 - 3 * alp, J1p=1 - alp, K1p=1 - 3 * alp, J1pp=1 - alp, K1pp=1 - 3 * alp)


def field_111(h: float) -> np.ndarray:
    """Field vector of magnitude h along [111]."""
    return np.full(3, h / math.sqrt(3.0))
