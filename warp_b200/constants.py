"""Physical constants with the values the reference uses
(pywarp90/top.v:170-190, 2010 CODATA; eps0 = 1/(mu0 c^2), top.F:380-384;
proton mass from scripts/species.py:174)."""
import math

pi = 3.14159265358979323
clight = 2.99792458e+8
echarge = 1.602176565e-19
amu = 1.660538921e-27
emass = 9.10938291e-31
mu0 = 4. * pi * 1.e-7
eps0 = 1. / (mu0 * clight * clight)
proton_mass = 1.6726231e-27
largepos = 1.0e36
smallpos = 1.0e-36


def beta_of_kinetic(ekin_ev, mass):
    """Relativistic beta of a particle with kinetic energy ekin_ev (eV)."""
    gamma = 1. + ekin_ev * echarge / (mass * clight * clight)
    return math.sqrt(1. - 1. / (gamma * gamma))
