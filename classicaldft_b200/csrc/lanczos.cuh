// Block Lanczos for the lowest eigenpair of the fixed-boundary Hessian of
// Omega, driven by the exact Hessian-vector products of an Engine.
//
// The reference finds the smallest eigenpair with a 3-vector Rayleigh-Ritz
// iteration on a finite-difference product (EigenvalueSolver::solve,
// include/dft/algorithms/saddle_point.hpp:171-276); its operator is the
// Hessian with the force rows of the boundary faces zeroed (:377-384).  This
// solver keeps that operator, restricted to the interior: every basis vector
// has zero faces, so the operator P H P (P zeroes the faces) is symmetric and
// its eigenvectors with non-zero eigenvalue are those of the reference's P H.
//
// Per iteration: one batched product W = A Q_j of the `block` directions of
// the current block (one launch sequence of the product engine, whose batch
// equals the block size), full re-orthogonalisation against the basis by two
// passes of block classical Gram-Schmidt, and a two-pass Cholesky QR of the
// remainder giving the next block and its coupling R_j.  Every inner product
// is a deterministic device reduction and stays on the device: the host reads
// the projected matrix only every `check_interval` iterations to solve the
// small symmetric eigenproblem and test the residual |R_j s_j| of the lowest
// Ritz pair.  When the basis is full the search restarts from the `block`
// lowest Ritz vectors.
#pragma once

#include "engine.cuh"

namespace cdft {

struct LanczosConfig {
  double tolerance = 1e-4;      // |A x - theta x| of the unit Ritz vector
  int max_iterations = 300;     // block products, restarts included
  int block = 1;                // directions per product (the product engine's batch)
  int max_basis = 32;           // blocks kept before a restart
  int check_interval = 4;       // iterations between host checks
  unsigned long long seed = 42; // random start vectors
};

struct LanczosResult {
  double eigenvalue = 0.0;  // x^T A x of the returned unit vector
  double residual = 0.0;    // |A x - eigenvalue x|
  int iterations = 0;       // block products (the final check product not counted)
  int restarts = 0;
  bool converged = false;
};

// Lowest eigenpair of the fixed-boundary Hessian at rho.  `hvp` evaluates the
// products (hvp_set_point / hvp_apply); its batch is the block size.  vec
// (device, N): start vector if use_guess (the other directions of the first
// block are drawn), receives the unit eigenvector (zero on the faces).
LanczosResult lanczos_lowest(Engine& hvp, const LanczosConfig& cfg, const double* rho, double* vec, bool use_guess,
                             cudaStream_t stream);

// Symmetric eigen-decomposition of the n x n row-major matrix a (cyclic
// Jacobi; host).  Eigenvalues ascending into w, eigenvectors as the columns
// of v (row-major n x n).
void symmetric_eigen(int n, const double* a, double* w, double* v);

}  // namespace cdft
