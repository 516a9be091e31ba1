// FP64 instantiation of the solver (the parity path and the mixed path's FP64
// fields).  The FP32 helper it creates for the mixed path is the instantiation
// compiled in solver_f32.cu.
#include "solver.cuh"

namespace vsav {

extern template class Solver<float>;
template class Solver<double>;

SolverBase* make_solver_f64(const Dims& d, const Phys& p, const Options& o, const int* run_sizes, const double* psi_in,
                            const double* psi_out) {
  return new Solver<double>(d, p, o, run_sizes, psi_in, psi_out);
}

}  // namespace vsav
