// host_check.cpp -- the product's per-root secular state machine
// (brdc_secular.cuh) compiled for the host, so the CPU test suite can check
// its numerics against LAPACK DLAED4 without a GPU.  Not used by the solver.
#include <cfloat>

#include "brdc_secular.cuh"

extern "C" int brdc_host_secular_root(int K, const double *d, const double *z,
                                      double rho, double znorm2, int i,
                                      int *org, double *tau, int *failed) {
    return brdc::sec_solve_serial(K, d, z, rho, znorm2, i, org, tau, failed,
                                  DBL_EPSILON);
}

// The same with an iteration cap of its own (the failure path).
extern "C" int brdc_host_secular_root_capped(int K, const double *d, const double *z,
                                             double rho, double znorm2, int i, int max_iter,
                                             int *org, double *tau, int *failed) {
    return brdc::sec_solve_serial(K, d, z, rho, znorm2, i, org, tau, failed,
                                  DBL_EPSILON, max_iter);
}
