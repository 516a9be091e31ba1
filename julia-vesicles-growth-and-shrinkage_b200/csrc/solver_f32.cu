// FP32 instantiation of the solver (the FP32 bulk path and the FP32 psi helper
// of the mixed path), compiled on its own so the two precisions build in parallel.
#include "solver.cuh"

namespace vsav {

template class Solver<float>;

SolverBase* make_solver_f32(const Dims& d, const Phys& p, const Options& o, const int* run_sizes, const double* psi_in,
                            const double* psi_out) {
  return new Solver<float>(d, p, o, run_sizes, psi_in, psi_out);
}

}  // namespace vsav
