// caffeCaseInfo: parses case/case.info and case/initialConditions.info of the working
// directory and prints the device library's case record as one JSON line (a check of the
// input mapping that needs no GPU).  Usage: caffeCaseInfo simple|piso|ibpiso
#include <cstdio>
#include <cstring>
#include <iostream>

#include "Input.h"
#include "Solver.h"

int main(int argc, const char* argv[]) {
    int kind = CAFFE_PISO;
    if (argc > 1) kind = std::strcmp(argv[1], "simple") == 0 ? CAFFE_SIMPLE : (std::strcmp(argv[1], "ibpiso") == 0 ? CAFFE_IBPISO : CAFFE_PISO);
    try {
        Input input;
        caffe_case c = Solver::caseFromInput(input, kind);
        std::printf("{\"kind\": %d, \"bc_type\": [%d, %d, %d, %d, %d, %d], \"ref_vec\": [", c.kind, c.bc_type[0], c.bc_type[1], c.bc_type[2],
                    c.bc_type[3], c.bc_type[4], c.bc_type[5]);
        for (int f = 0; f < 6; ++f) std::printf("%s[%.17g, %.17g, %.17g]", f ? ", " : "", c.ref_vec[f][0], c.ref_vec[f][1], c.ref_vec[f][2]);
        std::printf("], \"ref_val\": [%.17g, %.17g, %.17g, %.17g, %.17g, %.17g]", c.ref_val[0], c.ref_val[1], c.ref_val[2], c.ref_val[3],
                    c.ref_val[4], c.ref_val[5]);
        std::printf(", \"rho\": %.17g, \"mu\": %.17g, \"time_accurate\": %d, \"omega_u\": %.17g, \"omega_p\": %.17g", c.rho, c.mu,
                    c.time_accurate, c.omega_u, c.omega_p);
        std::printf(", \"n_inner\": %d, \"n_pcorr\": %d, \"convection\": %d, \"nonorth\": %d, \"mom_method\": %d, \"p_method\": %d",
                    c.n_inner, c.n_pcorr, c.convection, c.nonorth, c.mom_method, c.p_method);
        std::printf(", \"mom_rtol\": %.17g, \"p_rtol\": %.17g, \"maxit\": %d, \"ib_radius\": %.17g, \"ib_center\": [%.17g, %.17g, %.17g]",
                    c.mom_rtol, c.p_rtol, c.maxit, c.ib_radius, c.ib_center[0], c.ib_center[1], c.ib_center[2]);
        std::printf(", \"u_init\": [%.17g, %.17g, %.17g], \"p_init\": %.17g, \"p_form\": %d}\n", c.u_init[0], c.u_init[1], c.u_init[2],
                    c.p_init, c.p_form);
    } catch (const char* e) {
        std::cerr << "Error: " << e << std::endl;
        return 1;
    }
    return 0;
}
