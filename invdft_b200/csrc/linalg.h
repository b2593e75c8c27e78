// Small dense FP64 linear algebra for the subspace (N <= 64) steps of the
// Chebyshev-filtered subspace iteration: Cholesky orthonormalisation and the
// Rayleigh-Ritz eigenproblem.  These are N x N problems solved on the host in
// microseconds; the N_dof-sized work stays on the GPU.
#pragma once
#include <cstdint>
#include <vector>

namespace invdft {

// Lower Cholesky factor of symmetric positive definite S (row-major). False if not SPD.
bool cholesky_lower(int n, const std::vector<double> &S, std::vector<double> &L);
// T = L^{-T} (upper triangular), row-major.
void lower_inverse_transpose(int n, const std::vector<double> &L, std::vector<double> &T);
// Cyclic Jacobi eigensolver of symmetric A: ascending eigenvalues w, eigenvectors
// as columns of V (row-major V[i*n+j] = component i of vector j), each column
// signed so that its largest-magnitude entry is positive.
void jacobi_eigh(int n, const std::vector<double> &A, std::vector<double> &w, std::vector<double> &V);

// Exactly reproducible pseudo-random numbers in [-0.5, 0.5) from 32-bit integer hashing.
double hash_uniform(uint64_t i, uint64_t salt);

// Fermi-Dirac helpers (dftUtils::getPartialOccupancy / getPartialOccupancyDer forms).
double partial_occupancy(double eig, double mu, double kT);
double partial_occupancy_der(double eig, double mu, double kT);
double fermi_energy(const std::vector<double> &eig, double n_electrons, double kT);

}  // namespace invdft
