"""Analysis results (PSSFSS.jl ``src/Outputs.jl:24-37``, ``:73-89``).

``Result`` carries the full GSM of the structure for one (steering, frequency) point
plus the end-region media and lattices, exactly the fields of the reference's struct.
"""
from dataclasses import dataclass

import numpy as np

from .gsms import GSM
from .layers import TE, TM


@dataclass
class Result:
    gsm: GSM
    steering: dict          # {"θ": deg, "ϕ": deg} or {"ψ₁": deg, "ψ₂": deg}
    beta00: np.ndarray      # radians/meter
    FGHz: float
    epsr_in: complex
    mur_in: complex
    beta1_in: np.ndarray
    beta2_in: np.ndarray
    epsr_out: complex
    mur_out: complex
    beta1_out: np.ndarray
    beta2_out: np.ndarray

    def __repr__(self):
        return f"Result: {self.FGHz} GHz, {self.steering}, GSM{self.gsm.s12.shape}"


def getsijmn(i, j, m, n, r):
    """Entry (m, n) (1-based, or TE/TM) of partition (i, j) of ``r.gsm`` (Outputs.jl:73)."""
    return r.gsm[(i, j)][int(m) - 1, int(n) - 1]


def s_parameters(results, i, j, m, n):
    """Vector of ``S{i}{j}(m,n)`` over a list of results."""
    return np.array([getsijmn(i, j, m, n, r) for r in results])
