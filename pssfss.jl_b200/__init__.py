"""B200-native periodic method-of-moments fill-and-solve (the PSSFSS.jl hot path).

Public API mirrors PSSFSS.jl: ``analyze``, ``Layer``, sheet constructors (``rectstrip``,
``meander``, ``pecsheet``, ``pmcsheet``), length units and ``Result``.  The hot path
(modal tables, face-pair integrals, matrix fill, LU, solves, basis transforms and modal
projection) runs in ``libpssfss_b200.so`` (CUDA, sm_100a) through its C ABI.
"""
from .analyze import analyze
from .elements import meander, pecsheet, pmcsheet, rectstrip
from .layers import TE, TM, Layer
from .outputs import Result, getsijmn, s_parameters
from .rwg import setup_rwg
from .sheets import RWGSheet, combine, recttri
from .units import Length, cm, inch, m, mil, mm

__all__ = ["analyze", "Layer", "TE", "TM", "rectstrip", "meander", "pecsheet", "pmcsheet", "Result",
           "getsijmn", "s_parameters", "setup_rwg", "RWGSheet", "recttri", "combine", "Length", "mm", "cm",
           "inch", "mil", "m"]
