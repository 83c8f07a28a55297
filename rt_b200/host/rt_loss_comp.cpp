// rt_loss_comp -- the reference's losses_comp program
// (efficiency/losses_comp.cpp:11-136) on the B200 engine.
//
//   rt_loss_comp rt_files_list result_filename
//
// For every ray-tracing result named in rt_files_list (whitespace-separated
// names, as rt_trace writes them) it writes one block {size_t N_lambda;
// double lambda[N_lambda]; double ratio[N_lambda]}: the fraction of each
// wavelength's rays that reached the detector, computed on the device from
// the file's wavelengths (rtb_loss_ratios).
//
// The list is read as the reference reads it: names are taken with >> until
// the stream reports end of file, so after the last name of a list that ends
// in a newline one more, failed, read leaves the last name in place and that
// file's block is written twice -- kept, so that the result files match.  A
// file without good rays stops the program (the reference's load_beam_data
// returns 7 for it, beam.cpp:861).  Exit codes: 500 usage, 2 any error.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "rtb.h"

namespace {

int fail(int code, const std::string& file) {
    std::cerr << "An error (code = " << code << ") occured while reading ray-tracing file " << file << std::endl;
    return 2;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 3) {
        std::cout << "Usage: rt_loss_comp rt_files_list result_filename\n";
        return 500;
    }
    std::ifstream rt_files(argv[1]);
    std::string filename;
    FILE* result = std::fopen(argv[2], "wb");
    if (!result) return fail(100, filename);
    double* d_lambda = nullptr;
    size_t cap = 0;
    int rc = 0;
    while (!rt_files.eof()) {
        rt_files >> filename;
        std::cout << "Processing " << filename << " ..." << std::endl;
        uint64_t n = 0, n_good = 0, n_lambda = 0;
        if (rtb_read_dat_header(filename.c_str(), &n, &n_good, &n_lambda) != RTB_OK) {
            rc = fail(1, filename);
            break;
        }
        if (n_good == 0) {
            rc = fail(7, filename);
            break;
        }
        std::vector<double> lambda(n);
        rtb_rays h{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, lambda.data(), nullptr, nullptr, (size_t)n};
        if (rtb_read_dat(filename.c_str(), &h) != RTB_OK) {
            rc = fail(2, filename);
            break;
        }
        if (n > cap) {
            if (d_lambda) cudaFree(d_lambda);
            d_lambda = nullptr;
            if (cudaMalloc(&d_lambda, n * sizeof(double)) != cudaSuccess) {
                rc = fail(300, filename);
                break;
            }
            cap = n;
        }
        std::vector<double> ll(n_lambda), ratio(n_lambda);
        if (cudaMemcpy(d_lambda, lambda.data(), n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
            rtb_loss_ratios(d_lambda, n, n_good, n_lambda, ll.data(), ratio.data(), nullptr) != RTB_OK) {
            rc = fail(300, filename);
            break;
        }
        const size_t nl = (size_t)n_lambda;
        if (std::fwrite(&nl, sizeof(size_t), 1, result) != 1 || std::fwrite(ll.data(), 8, nl, result) != nl ||
            std::fwrite(ratio.data(), 8, nl, result) != nl) {
            rc = fail(200, filename);
            break;
        }
    }
    if (d_lambda) cudaFree(d_lambda);
    std::fclose(result);
    return rc;
}
