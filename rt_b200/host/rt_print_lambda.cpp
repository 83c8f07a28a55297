// rt_print_lambda -- the reference's print_lambda tool (tools/print_lambda.cpp)
// on the B200 engine.
//
//   rt_print_lambda rt_list_filename
//
// For every ray-tracing result named in the list (one per line; a last line
// without a newline is not read, as in the reference) it prints "# <name>",
// the distinct wavelengths of the good rays in order of first occurrence
// with 9 decimals, and an empty line.  The distinct values are found on the
// device (rtb_unique_lambdas).  The reference stops listing when the count of
// distinct values reaches the file's N_lambda at the end of a step, starting
// from the first good ray's value: with N_lambda >= 2 that caps the list at
// N_lambda values; with N_lambda 1 only when the second good ray repeats the
// first (or there is no second), and with N_lambda 0 never -- the same here.
// Exit codes: 1 usage or list error, 10 a file that cannot be read.
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "rtb.h"

int main(int argc, char** argv) {
    if (argc < 2) {
        std::cerr << "Usage: rt_print_lambda rt_list_filename\n";
        return 1;
    }
    std::cout << std::fixed << std::setprecision(9);
    std::ifstream rt_files(argv[1]);
    int flag = 0;
    std::string name;
    double* d_lambda = nullptr;
    size_t cap = 0;
    while (!rt_files.eof()) {
        std::getline(rt_files, name);
        if (rt_files.eof()) break;
        if (rt_files.fail() || rt_files.bad()) {
            std::cerr << "\nAn error occured while read the RT-list file!!!\n";
            flag = 1;
            break;
        }
        uint64_t n = 0, n_good = 0, n_lambda = 0;
        if (rtb_read_dat_header(name.c_str(), &n, &n_good, &n_lambda) != RTB_OK || n_good == 0) {
            flag = 10;
            break;
        }
        std::vector<double> lambda(n);
        rtb_rays h{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, lambda.data(), nullptr, nullptr, (size_t)n};
        if (rtb_read_dat(name.c_str(), &h) != RTB_OK) {
            flag = 10;
            break;
        }
        uint64_t max_out = n_lambda;
        if (n_lambda == 0 || (n_lambda == 1 && n_good > 1 && !(lambda[1] == lambda[0]))) max_out = n_good;
        if (n_good > cap) {
            if (d_lambda) cudaFree(d_lambda);
            d_lambda = nullptr;
            if (cudaMalloc(&d_lambda, n_good * sizeof(double)) != cudaSuccess) {
                flag = 10;
                break;
            }
            cap = n_good;
        }
        std::vector<double> uniq(max_out);
        uint64_t n_uniq = 0;
        if (cudaMemcpy(d_lambda, lambda.data(), n_good * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
            rtb_unique_lambdas(d_lambda, n_good, max_out, uniq.data(), &n_uniq, nullptr) != RTB_OK) {
            flag = 10;
            break;
        }
        std::cout << "# " << name << std::endl;
        for (uint64_t k = 0; k < n_uniq; ++k) std::cout << uniq[k] << std::endl;
        std::cout << "\n";
    }
    if (d_lambda) cudaFree(d_lambda);
    return flag;
}
