// Physical constants of src/constants/constants.h (mir-group/phoebe), usable
// from host and device code.
#pragma once
namespace phxc {
constexpr double pi = 3.14159265358979323846;
constexpr double twoPi = 2.0 * pi;
constexpr double sqrtPi = 1.7724538509055160273;  // sqrt(pi)
constexpr double hPlanckSi = 6.62607015e-34;
constexpr double hartreeSi = 4.359744650e-18;
constexpr double speedLightSi = 299792458.0;
constexpr double electronVoltSi = 1.6021766208e-19;
constexpr double rydbergSi = hartreeSi / 2.0;
constexpr double energyRyToEv = rydbergSi / electronVoltSi;
constexpr double TeraHertzAu = hPlanckSi / twoPi / hartreeSi * 1.0e12;
constexpr double ryToTHz = 1.0 / TeraHertzAu / 2.0 / twoPi;
constexpr double ryToCmm1 = 1.0e10 * ryToTHz / speedLightSi;
// delta_function.h:107,137
constexpr double adaptiveCutoff = 0.0001 / energyRyToEv;
constexpr double erf2 = 0.9953222650189527;
// ph_scattering.cpp:66, scattering.cpp:37, phonon_h0.cpp:1012
constexpr double phEnergyCutoff = 0.001 / ryToCmm1;
constexpr double phExcludeCutoff = 0.1 / ryToCmm1;
constexpr double velDegThreshold = 0.0001 / ryToCmm1;
constexpr double degThreshold = 1.0e-6;
// el_scattering.cpp:127
constexpr double elPhononCutoff = 5.0 / ryToCmm1;
}  // namespace phxc
