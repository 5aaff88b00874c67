#pragma once
// Solver options (fields and defaults of the reference's
// include/vikalp/contracts/SolverOptions.hpp:7-28), plus `b200`, the
// library-specific extension (scheme, precision, product order); its defaults
// reproduce the reference scheme.
#include "vikalp/contracts/Model.hpp"

namespace vikalp {

enum class BackendPreference { Auto, CPU, CUDA };
enum class ContinuousMethod { Auto, PDHG, RevisedSimplex, InteriorPoint };

// The B200 path's own knobs (no reference counterpart).
struct B200Options {
    enum class Scheme { Reference, Halpern } scheme = Scheme::Reference;
    bool mixed_precision = false;          // Halpern only: float32 iterates, float64 reductions / polish
    bool sequential_products = false;      // bit-identical sums in the reference CPU order
    Scalar relative_tolerance = 1e-6;      // Halpern stop: relative KKT in original units
    int check_every = 64;
    int device = 0;
};

struct SolverOptions {
    BackendPreference backend = BackendPreference::Auto;
    ContinuousMethod continuous_method = ContinuousMethod::Auto;
    Index iteration_limit = 100'000;
    Index node_limit = 100'000;
    Scalar time_limit_seconds = Model::infinity();
    // Feasibility and KKT residual limits in original, unscaled coordinates.
    Scalar primal_tolerance = 1e-7;
    Scalar dual_tolerance = 1e-7;
    Scalar integrality_tolerance = 1e-6;
    Scalar absolute_gap_tolerance = 1e-6;
    Scalar relative_gap_tolerance = 1e-4;
    bool deterministic = true;
    B200Options b200;
};

} // namespace vikalp
