// Device state of the conjugate-gradient solvers.
#pragma once

#include "spmv.cuh"
#include "space.cuh"

namespace ciecu {

// Scalars of ConjugateGradients_impl.hpp:49-201 kept on the device so an
// iteration never waits for the host.
struct PcgScalars {
    double rz;          // r^T z of the current iteration (preconditionedNorm)
    double pq;          // p^T A p
    double alpha;       // searchScale
    double beta;        // rz_new / rz_old
    double rr;          // r^T r (residualNorm)
    double r0;          // ||r_0||
    double absres;      // ||r||
    double relres;      // ||r|| / ||r_0||
    long long iter;     // loop index (iterationCount)
    long long maxIter;
    double absTol, relTol;
    int done;           // 0 running, 1 converged, 2 iteration limit, 3 error
    int error;          // 0, CIECU_ERR_BREAKDOWN
    long long errorIter;
    int errorKind;      // 1: r^T z <= 0 at start, 2: p^T A p <= 0
    int pad;
    long long chunkIter;   // iterations run by the current graph launch
    long long chunkLimit;  // iterations one graph launch may run
};

// Comparison::less with the default tolerances
// (cieutils/packages/maths/impl/Comparison_impl.hpp:32-63).
__device__ __forceinline__ bool float_less(double a, double b) {
    double norm = fabs(a) + fabs(b);
    norm = fmin(norm, 1.7976931348623157e308);
    const double tol = fmax(2.2250738585072014e-308, 2.220446049250313e-16 * norm);
    return a < b && !(fabs(a - b) < tol);
}

}  // namespace ciecu
