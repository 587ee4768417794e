// solver_fast.cu — the fast build of the Gauss-Seidel solver.
//
// solver.cuh compiled with FMA contraction and approximate division and square
// root (-fmad=true -prec-div=false -prec-sqrt=false; denormals kept): every
// projection, contact solve and solver kernel of the IEEE build in step_kernels.cu,
// in the same order and launch shapes, with shorter dependent arithmetic
// chains. Each operation differs from the IEEE result by a few ulp at most, so a
// projection's result stays within 1e-5 relative of the reference's (checked
// against the CPU oracle by the GPU tests); detection is not compiled here and
// stays bit-exact.
#include "step_common.cuh"
#include <cooperative_groups.h>
#include <cstdio>
#include <mutex>

namespace cg = cooperative_groups;

namespace sc {
namespace fast {
#include "solver.cuh"
} // namespace fast

const SolverOps& solver_ops_fast() { return fast::kSolverOps; }

} // namespace sc
