"""Physical constants of the reference (``Source/Constants.f90:50-79``)."""
import math

PI = 3.141592653589793238462643
Q_ELEC = 1.602176462e-19           # C
LIGHT = 299792458.0                # m/s
BOHR = 0.529177208607388           # Angstrom
M_TO_A = 1.0e10
MU0 = 4.0 * PI * 1.0e-7
EPS0 = 1.0 / (MU0 * LIGHT ** 2)
# Hartree -> eV exactly as derived in Source/Constants.f90:74
HARTREE_TO_EV = Q_ELEC * M_TO_A / (4.0 * PI * EPS0 * BOHR)
MACH_PREC = 2.220446049250313e-16  # printed by the reference (sample.output:15)

# Thomas-Fermi constant (Source/KEDF_TF.f90:42)
C_TF = 2.87123400018819

SQRT_MACH = math.sqrt(MACH_PREC)
