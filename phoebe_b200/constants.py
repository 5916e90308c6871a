"""Physical constants and unit conversions, with the values Phoebe uses.

Values follow src/constants/constants.h:1-71 of mir-group/phoebe, including
its quirk that ``fourPi`` equals 2*pi (constants.h:12).  Every quantity on the
scattering-rate path is in Rydberg atomic units: energies in Ry (hbar = 1),
lengths in Bohr, masses in Ry mass units (electron mass / 2).
"""
import math

pi = 3.14159265358979323846
sqrtPi = math.sqrt(pi)
twoPi = 2.0 * pi
fourPi = 2.0 * pi  # constants.h:12 (sic)

speedLightSi = 299792458.0
electronSi = 1.602176487e-19
hPlanckSi = 6.62607015e-34
hBarSi = hPlanckSi / twoPi
electronVoltSi = 1.6021766208e-19
hartreeSi = 4.359744650e-18
bohrRadiusSi = 0.52917721067e-10
rydbergSi = hartreeSi / 2.0
timeRy = hBarSi / rydbergSi
kBoltzmannSi = 1.38064852e-23
kBoltzmannRy = kBoltzmannSi / rydbergSi
electronMassSi = 9.10938215e-31
amuSi = 1.660538782e-27

temperatureAuToSi = 1.0 / kBoltzmannRy
energyRyToEv = rydbergSi / electronVoltSi
distanceAngToSi = 1.0e-10
distanceRyToSi = bohrRadiusSi
distanceBohrToAng = bohrRadiusSi / distanceAngToSi
timeAuToFs = timeRy * 1e15
energyRyToFs = timeAuToFs * twoPi
massAmuToRy = amuSi / electronMassSi / 2.0
massRyToAmu = 1.0 / massAmuToRy

TeraHertzAu = hPlanckSi / twoPi / hartreeSi * 1.0e12
ryToTHz = 1.0 / TeraHertzAu / 2.0 / twoPi
ryToCmm1 = 1.0e10 * ryToTHz / speedLightSi
velocityRyToSi = distanceRyToSi * rydbergSi / hBarSi
thConductivityAuToSi = kBoltzmannSi * rydbergSi / bohrRadiusSi / hBarSi

# delta_function.h:107,137 -- adaptive smearing floor and erf(2)
adaptiveBroadeningCutoff = 0.0001 / energyRyToEv
erf2 = 0.9953222650189527

# ph_scattering.cpp:66, scattering.cpp:37 -- low-energy cutoffs
phEnergyCutoff = 0.001 / ryToCmm1
phExcludeCutoff = 0.1 / ryToCmm1
# scattering.cpp:1190,1223 -- degeneracy threshold on energies (Ry)
degeneracyThreshold = 1.0e-6
# phonon_h0.cpp:1012 -- velocity degenerate-subspace threshold
velocityDegeneracyThreshold = 0.0001 / ryToCmm1


def kelvin_to_ry(t_kelvin):
    """Temperature in K -> Ry (context.cpp:537 divides by temperatureAuToSi)."""
    return t_kelvin / temperatureAuToSi
