"""Physical constants and fixed algorithm parameters.

Mirrors PSSFSS.jl ``src/Constants.jl:5-28``; every value is the same IEEE double the
reference builds (``μ₀ = 1.25663706212e-6``, ``ϵ₀ = 1/(μ₀ c₀²)``, ...).
"""
import math

MU0 = 1.25663706212 * 1e-6          # Constants.jl:6
C0 = 299792458.0                     # Constants.jl:9
EPS0 = 1.0 / (MU0 * C0 ** 2)         # Constants.jl:12
ETA0 = math.sqrt(MU0 / EPS0)         # Constants.jl:15
TWOPI = 2.0 * math.pi                # Constants.jl:17
FOURPI = 4.0 * math.pi               # Constants.jl:18
TOL = 1e-4                           # Constants.jl:19 (J/K cache relative tolerance on u)
DBMIN = 30.0                         # Constants.jl:22
MIN_ELENGTH = TWOPI * 0.1            # Constants.jl:25

# Spectral / spatial series controls (PGF.jl:15,18,217; FillZY.jl:69,293)
JKRINGMAX = 65
MMAX_LIST = (32, 2048)
CONVREPEAT = 40
TABLE_CONVTEST = 1e-7
JK_CONVTEST = 1e-8
UFACTOR = 0.5                        # PSSFSS.jl:224
