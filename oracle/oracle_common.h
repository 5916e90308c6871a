// CPU FP64 oracle for the scattering-rate path of mir-group/phoebe.
//
// TEST INFRASTRUCTURE ONLY.  This library restates the reference's CPU
// algorithms so that the CUDA product can be checked against them.  Only the
// test suite, the smoke check and the CPU-baseline leg of the benchmark load
// it; the product library never links, loads or calls it.
//
// Conventions shared by all oracle entry points:
//   * arrays are C-order (row-major) in the reference's index order;
//   * complex arrays are interleaved (re, im) doubles;
//   * eigenvector matrices are U[a][b]: row a = 3*atom + cartesian,
//     column b = band (the columns of Eigen's eigenvector matrix);
//   * energies/frequencies in Ry, lengths in Bohr, masses in Ry units.
#pragma once
#include <complex>
#include <vector>
#include <cmath>

namespace orc {

using cd = std::complex<double>;

// src/constants/constants.h:1-71 (values as the reference defines them)
constexpr double pi = 3.14159265358979323846;
constexpr double twoPi = 2.0 * pi;
const double sqrtPi = std::sqrt(pi);
constexpr double hPlanckSi = 6.62607015e-34;
constexpr double hartreeSi = 4.359744650e-18;
constexpr double speedLightSi = 299792458.0;
constexpr double electronVoltSi = 1.6021766208e-19;
constexpr double rydbergSi = hartreeSi / 2.0;
constexpr double energyRyToEv = rydbergSi / electronVoltSi;
const double TeraHertzAu = hPlanckSi / twoPi / hartreeSi * 1.0e12;
const double ryToTHz = 1.0 / TeraHertzAu / 2.0 / twoPi;
const double ryToCmm1 = 1.0e10 * ryToTHz / speedLightSi;

// Hermitian eigen-decomposition (Householder tridiagonalisation + implicit
// QL), ascending eigenvalues.  A is n*n row-major, overwritten.  Vectors in
// columns of Z (row-major).  Returns 0 on success.
int hermitian_eig(int n, cd* A, double* w, cd* Z);

}  // namespace orc
