// rt_ccd_frame -- the reference's ccd_frame program (ccd/ccd_frame.cpp:21-321)
// on the B200 engine.
//
//   rt_ccd_frame rt_files_list QE_filename spec_filename ccd_spec_filename result_FITS_filename
//
// For every .dat file named in rt_files_list (one per line, as rt_trace
// writes them) it reads the next block of the QE file ({size_t N; double
// lambda[N]; double QE[N]}, one block per file, scheme.cpp:1115-1121), puts
// the good rays on the CCD (rtb_ccd_coordinates) and adds
// spec(lambda) * lambda / hc * QE(lambda) * pixel area per ray to the image
// (rtb_compute_ccd_image); the image is written as a FITS DOUBLE image with
// the keywords RT_LIST, QE_FILE, SPECFILE and CCDINFO (rtb_write_fits).  The
// CCD file holds three data lines: linear size x y (mm), pixels x y, pixel
// size x y (mm); '#' starts a comment line.  Exit codes follow the
// reference: 1 usage, 2 CCD file, 3 QE or spectrum file, 4 FITS, 5 list or
// ray-tracing file, 100 memory.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "rtb.h"

namespace {

// AsciiFile::ReadLine (common-lib/ascii_file.cpp): blank and '#' lines are
// skipped; `need` numbers must start a data line.  Returns 1 for a data line,
// 0 at end of file, -1 for an invalid line.  A last line without a newline
// is not read, as in the reference.
int read_line(std::ifstream& f, size_t need, std::vector<double>& v) {
    std::string line;
    for (;;) {
        if (!std::getline(f, line) || f.eof()) return 0;
        size_t k = 0;
        while (k < line.size() && line[k] == ' ') ++k;
        if (k == line.size() || line[k] == '#') continue;
        const char* p = line.c_str() + k;
        v.clear();
        for (size_t j = 0; j < need; ++j) {
            char* e = nullptr;
            double x = std::strtod(p, &e);
            if (e == p) return -1;
            v.push_back(x);
            p = e;
        }
        return 1;
    }
}

struct Table {
    std::vector<double> x, y, y2;
    rtb_table t{};
    bool set(std::vector<double> xs, std::vector<double> ys) {
        x = std::move(xs);
        y = std::move(ys);
        if (x.size() < 4) return false;
        for (size_t k = 1; k < x.size(); ++k)
            if (!(x[k] > x[k - 1])) return false;
        y2.assign(x.size(), 0.0);
        if (rtb_spline_init(x.size(), x.data(), y.data(), y2.data()) != RTB_OK) return false;
        t.n = x.size();
        t.x = x.data();
        t.y = y.data();
        t.y2 = y2.data();
        return true;
    }
};

}  // namespace

int main(int argc, char** argv) {
    if (argc < 6) {
        std::cerr << "Usage: rt_ccd_frame rt_files_list QE_filename spec_filename ccd_spec_filename "
                     "result_FITS_filename\n";
        return 1;
    }
    double xsize, ysize, xdimf, ydimf, xpix, ypix;
    {
        std::ifstream f(argv[4]);
        if (!f) {
            std::cerr << "Can not open CCD specification file!\n";
            return 2;
        }
        std::vector<double> v;
        double* dst[3][2] = {{&xsize, &ysize}, {&xdimf, &ydimf}, {&xpix, &ypix}};
        for (auto& d : dst) {
            if (read_line(f, 2, v) != 1) {
                std::cerr << "Invalid CCD linear size specification!\n";
                return 2;
            }
            *d[0] = v[0];
            *d[1] = v[1];
        }
    }
    const size_t xdim = (size_t)xdimf, ydim = (size_t)ydimf;
    std::cout << "CCD specifications:\nLinear size: [" << xsize << ":" << ysize << "]\nPixel linear size: [" << xpix
              << ":" << ypix << "]\nNumber of pixels: [" << xdim << ":" << ydim << "]\n";
    FILE* qe_file = std::fopen(argv[2], "rb");
    if (!qe_file) {
        std::cerr << "Can not open QE file!\n";
        return 3;
    }
    Table spec;
    {
        std::ifstream f(argv[3]);
        std::vector<double> xs, ys, v;
        int r;
        while ((r = read_line(f, 2, v)) == 1) {
            xs.push_back(v[0]);
            ys.push_back(v[1]);
        }
        if (!f.is_open() || r < 0 || !spec.set(xs, ys)) {
            std::cerr << "Can not load input spectrum function!\n";
            std::fclose(qe_file);
            return 3;
        }
    }
    std::vector<double> image;
    try {
        image.assign(xdim * ydim, 0.0);
    } catch (...) {
        std::cerr << "Can not allocate memory for the result image!\n";
        std::fclose(qe_file);
        return 100;
    }
    std::ifstream list(argv[1]);
    if (!list) {
        std::cerr << "Can not open file with list of ray-tracing result files!\n";
        std::fclose(qe_file);
        return 5;
    }
    std::cout << "\nSTART CCD IMAGE CREATION ...\n";
    std::string fn;
    int rc = 0;
    uint64_t outside_total = 0;
    while (std::getline(list, fn)) {
        if (list.eof()) break;  // the reference stops before an unterminated last line
        std::cout << "   Processing file: " << fn << "...  \n";
        size_t npts = 0;
        Table qe;
        if (std::fread(&npts, sizeof(size_t), 1, qe_file) != 1) {
            std::cerr << "\nAn error occured while read QE file!\n";
            rc = 5;
            break;
        }
        std::vector<double> ql(npts), qv(npts);
        if (std::fread(ql.data(), sizeof(double), npts, qe_file) != npts ||
            std::fread(qv.data(), sizeof(double), npts, qe_file) != npts || !qe.set(ql, qv)) {
            std::cerr << "\nAn error occured while read QE file!\n";
            rc = 5;
            break;
        }
        uint64_t n = 0, ng = 0, nl = 0;
        if (rtb_read_dat_header(fn.c_str(), &n, &ng, &nl) != RTB_OK) {
            std::cerr << "\nAn error occured while read the ray-tracing output file!\n";
            rc = 5;
            break;
        }
        std::vector<double> a[7];
        for (auto& v : a) v.assign(n, 0.0);
        rtb_rays hr{a[0].data(), a[1].data(), a[2].data(), a[3].data(), a[4].data(), a[5].data(), a[6].data(),
                    nullptr, nullptr, (size_t)n};
        if (rtb_read_dat(fn.c_str(), &hr) != RTB_OK) {
            std::cerr << "\nAn error occured while read the ray-tracing output file!\n";
            rc = 5;
            break;
        }
        std::vector<unsigned> cx(ng ? ng : 1), cy(ng ? ng : 1);
        if (rtb_ccd_coordinates(ng, a[0].data(), a[1].data(), xsize, ysize, xpix, ypix, cx.data(), cy.data()) !=
            RTB_OK) {
            std::cerr << "\nAn error occured while compute CCD coordinates!\n";
            rc = 5;
            break;
        }
        uint64_t outside = 0;
        if (rtb_compute_ccd_image(ng, cx.data(), cy.data(), a[6].data(), &qe.t, &spec.t, xdim, ydim, xpix, ypix,
                                  image.data(), &outside) != RTB_OK) {
            std::cerr << "\nAn error occured while compute CCD image!\n";
            rc = 5;
            break;
        }
        outside_total += outside;
    }
    std::fclose(qe_file);
    if (rc) return rc;
    std::cout << "DONE!  (" << outside_total << " good rays fell outside the CCD)\n\nSAVE IMAGE TO FITS FILE ...  ";
    const char* keys[4] = {"RT_LIST", "QE_FILE", "SPECFILE", "CCDINFO"};
    const char* vals[4] = {argv[1], argv[2], argv[3], argv[4]};
    if (rtb_write_fits(argv[5], image.data(), xdim, ydim, keys, vals, 4) != RTB_OK) {
        std::cerr << "Can not create result FITS file!\n";
        return 4;
    }
    std::cout << "OK!\n";
    return 0;
}
