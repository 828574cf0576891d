// Driver-side view of the stand-in PETSc (test infrastructure): the tolerance of its tight
// solve and the record of every system the reference's code handed to KSPSolve.
#ifndef CAFFE_REFSHIM_H
#define CAFFE_REFSHIM_H

#include <vector>

namespace refshim {

struct System {
    int n = 0;
    std::vector<int> ptr, col;   // CSR of the rows as assembled (columns ascending)
    std::vector<double> val, b, x;
};

void set_solve_tolerance(double rtol, int maxit);
void set_recording(bool on);
std::vector<System>& systems();
// solutions for the next KSPSolve calls, in order (each call takes the next one instead of solving)
void inject(const double* x, int n);
void clear_injected();
int injected_left();

}  // namespace refshim

#endif
