"""Physical constants, CODATA 2018, as the reference defines them (src/MaxwellFDTD.jl:17-23)."""
import math

C0 = 299792458.0                 # SpeedOfLightInVacuum
EPS0 = 8.8541878128e-12          # VacuumElectricPermittivity
MU0 = 1.25663706212e-6           # VacuumMagneticPermeability
QE = 1.602176634e-19             # ElementaryCharge
ME = 9.1093837015e-31            # ElectronMass
HBAR = 6.62607015e-34 / (2 * math.pi)   # ReducedPlanckConstant = h / 2pi (1.0545718176461565e-34)
