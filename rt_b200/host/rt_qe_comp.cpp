// rt_qe_comp -- the reference's qe_comp program (efficiency/efficiency.cpp
// with Scheme::ComputeQE, common-lib/scheme.cpp:1123-1338) on the B200 engine.
//
//   rt_qe_comp scheme_file number_of_wavelengths result_file
//
// Loads the scheme file (rtb_scheme_load), takes its QE surfaces (every
// non-AUX MIRROR, LENS, GRATING and DETECTOR with its qe_curve, gratings with
// their blaze parameters: rtb_scheme_qe_surfaces) and computes, for every
// wavelength range, the throughput at number_of_wavelengths equally spaced
// wavelengths from w1 to w2 -- the product of the surfaces' QE curves and the
// gratings' blaze efficiency in their orders (rtb_qe_curves, one launch for
// all ranges).  The result file holds one block per range, {size_t N;
// double lambda[N]; double QE[N]}, the file rt_ccd_frame reads.
//
// The reference prints the SchemeError of a failing scheme and exits 0; here
// a failure exits 2 (scheme), 3 (computation) or 4 (result file), and a
// usage error or a number of wavelengths that is not an integer >= 2 exits 1.
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <vector>

#include "rtb.h"

int main(int argc, char** argv) {
    if (argc < 4) {
        std::cerr << "Usage: rt_qe_comp scheme_file number_of_wavelengths result_file\n";
        return 1;
    }
    char* end = nullptr;
    const long long nl = std::strtoll(argv[2], &end, 10);
    if (end == argv[2] || *end != '\0' || nl < 2) {
        std::cerr << "rt_qe_comp: the number of wavelengths must be an integer >= 2\n";
        return 1;
    }
    const size_t n_lambda = (size_t)nl;
    std::cout << "Load scheme file ...";
    rtb_scheme* sc = nullptr;
    int serr = -1;
    if (rtb_scheme_load(argv[1], &sc, &serr) != RTB_OK) {
        std::cout << "\nSomething is wrong!\nError: " << serr << "\n";
        return 2;
    }
    std::cout << "  OK!\n";
    const rtb_qe_surface* qs = nullptr;
    size_t n_qs = 0;
    if (rtb_scheme_qe_surfaces(sc, &qs, &n_qs, &serr) != RTB_OK) {
        std::cout << "\nSomething is wrong!\nError: " << serr << "\n";
        rtb_scheme_free(sc);
        return 2;
    }
    const double* rows = nullptr;
    size_t n_rows = 0, row_len = 0;
    rtb_scheme_ranges(sc, &rows, &n_rows, &row_len);
    std::cout << "Compute QE curve ...";
    std::vector<double> lambda(n_rows * n_lambda), qe(n_rows * n_lambda);
    int st = rtb_qe_curves(qs, n_qs, rows, n_rows, row_len, n_lambda, lambda.data(), qe.data());
    rtb_scheme_free(sc);
    if (st != RTB_OK) {
        std::cout << "\nSomething is wrong!\nError: engine status " << st << "\n";
        return 3;
    }
    if (rtb_save_qe(argv[3], n_rows, n_lambda, lambda.data(), qe.data()) != RTB_OK) {
        std::cout << "\nSomething is wrong!\nError: can not write " << argv[3] << "\n";
        return 4;
    }
    std::cout << "  OK!\n";
    return 0;
}
