// Covariance-parameter estimation by minimum contrast
// (estimate_kernel_parameters.h): the lattice offsets and their distances,
// and the constrained least-squares fit of the RBF covariance to the
// summary, minimised with COBYLA.
#pragma once

#include <functional>
#include <string>
#include <vector>

namespace drb {

// perturbation_matrix_3d (perturbation_matrix.h:62-109): 3 ints per offset.
std::vector<int> mce_offsets();

// |(P, 0) Q^T| row norms in float ((P.cast<float>() * Q.transpose()).rowwise().norm()).
std::vector<float> mce_distances(const std::vector<int>& P, const float* Q);

// COBYLA (Powell 1994, "A direct search optimization method that models the
// objective and constraint functions by linear interpolation"): minimises
// f(x) subject to c_k(x) >= 0.  `step` is the initial simplex edge per
// variable (the problem is solved in coordinates scaled by it), `rho_end` the
// final trust-region radius in those coordinates.  Returns the number of
// evaluations; x holds the best point found.
int cobyla_minimize(int n, int m, std::vector<double>& x, const std::vector<double>& step, double rho_end,
                    int max_eval, const std::function<double(const double*, double*)>& fc);

// compute_rbf_parameters (estimate_kernel_parameters.h:267-390) with its
// defaults: constrained (bandwidth <= exponent), no distance cut, no fixed
// parameters, xtol 1e-5.  theta: start values in, estimate out.
// Returns 0, or 1 when the fit cannot be run (the reference's retval).
int fit_rbf_parameters(const float* distance, const float* covariance, const int* npairs, int n, double* theta,
                       std::string* err);

}  // namespace drb
