// io.cu -- the reference's result files: .dat beams and FITS images.
//
// .dat (Beam::Save, common-lib/beam.cpp:636-715): size_t Nrays, N_good,
// N_lambda; the seven arrays X Y Z cX cY cZ lambda of the good rays, each
// contiguous; then the seven arrays of the lost rays.  Rays appear in the
// order the reference's Rearrange calls leave them, which rtb_reference_order
// replays; rtb_save_dat gathers a beam's rays in that order on the device,
// copies them to page-locked memory and writes the file.
//
// FITS (ccd/ccd_frame.cpp:263-314 writes through CFITSIO): one primary HDU,
// 2880-byte blocks of 80-character header cards, then the image as big-endian
// IEEE doubles (BITPIX = -64, the reference's DOUBLE_IMG), padded with zeros
// to a whole block.  Written here directly from the FITS standard.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "engine.cuh"

namespace rtb {
namespace {

__global__ void k_gather_beam(DevRays r, const uint32_t* order, uint64_t first, uint64_t n, double* out) {
    const double* src[7] = {r.X, r.Y, r.Z, r.cX, r.cY, r.cZ, r.lambda};
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = first + order[first + k];
#pragma unroll
        for (int c = 0; c < 7; ++c) out[(uint64_t)c * n + k] = src[c][i];
    }
}

bool put(FILE* f, const void* p, size_t bytes) { return bytes == 0 || std::fwrite(p, 1, bytes, f) == bytes; }

std::string card(const std::string& key, const std::string& value, const std::string& comment = "") {
    char buf[81];
    if (key == "END") {
        std::snprintf(buf, sizeof(buf), "%-80s", "END");
    } else {
        std::string v = value;
        std::string c = comment.empty() ? "" : " / " + comment;
        std::snprintf(buf, sizeof(buf), "%-8.8s= %20s%s", key.c_str(), v.c_str(), c.c_str());
    }
    std::string s(buf);
    s.resize(80, ' ');
    return s;
}

std::string fits_string(const char* s) {  // quoted, quotes doubled, at least 8 characters inside
    std::string o = "'";
    for (const char* p = s; *p && o.size() < 68; ++p) {
        o += *p;
        if (*p == '\'') o += '\'';
    }
    while (o.size() < 9) o += ' ';
    return o + "'";
}

}  // namespace
}  // namespace rtb

using namespace rtb;

extern "C" {

int rtb_save_dat(const char* path, const rtb_rays* rays, const uint32_t* order, uint64_t first, uint64_t n,
                 uint64_t n_good, uint64_t n_lambda, void* stream) {
    if (!path || !rays || (!order && n) || n_good > n || first + n > rays->n || !rays->lambda) return RTB_BAD_VALUE;
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : engine().stream;
    const size_t bytes = (size_t)7 * n * sizeof(double);
    DevBuf dbuf;
    double* host = nullptr;
    if (n) {
        if ((st = dbuf.alloc(bytes, s)) != RTB_OK) return st;
        RTB_CUDA_TRY(cudaMallocHost(&host, bytes));
        k_gather_beam<<<grid_for(n, 256, 8), 256, 0, s>>>(dev_rays(rays), order, first, n, dbuf.as<double>());
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(host, dbuf.p, bytes, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            cudaFreeHost(host);
            return cuda_status(e);
        }
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) {
        if (host) cudaFreeHost(host);
        return RTB_FAILED;
    }
    const size_t hdr[3] = {(size_t)n, (size_t)n_good, (size_t)n_lambda};
    bool ok = put(f, hdr, sizeof(hdr));
    for (int part = 0; part < 2 && ok; ++part) {  // good rays, then lost rays
        const uint64_t k0 = part ? n_good : 0, cnt = part ? n - n_good : n_good;
        for (int c = 0; c < 7 && ok; ++c) ok = put(f, host + (size_t)c * n + k0, cnt * sizeof(double));
    }
    ok = (std::fclose(f) == 0) && ok;
    if (host) cudaFreeHost(host);
    return ok ? RTB_OK : RTB_FAILED;
}

int rtb_read_dat_header(const char* path, uint64_t* n, uint64_t* n_good, uint64_t* n_lambda) {
    if (!path || !n || !n_good || !n_lambda) return RTB_BAD_VALUE;
    FILE* f = std::fopen(path, "rb");
    if (!f) return RTB_FAILED;
    size_t hdr[3];
    const bool ok = std::fread(hdr, sizeof(size_t), 3, f) == 3;
    std::fclose(f);
    if (!ok || hdr[1] > hdr[0]) return RTB_BAD_VALUE;
    *n = hdr[0];
    *n_good = hdr[1];
    *n_lambda = hdr[2];
    return RTB_OK;
}

int rtb_read_dat(const char* path, const rtb_rays* host_rays) {
    if (!path || !host_rays) return RTB_BAD_VALUE;
    FILE* f = std::fopen(path, "rb");
    if (!f) return RTB_FAILED;
    size_t hdr[3];
    bool ok = std::fread(hdr, sizeof(size_t), 3, f) == 3 && hdr[1] <= hdr[0] && hdr[0] == host_rays->n;
    double* dst[7] = {host_rays->X, host_rays->Y, host_rays->Z, host_rays->cX, host_rays->cY, host_rays->cZ,
                      host_rays->lambda};
    for (int part = 0; part < 2 && ok; ++part) {
        const size_t k0 = part ? hdr[1] : 0, cnt = part ? hdr[0] - hdr[1] : hdr[1];
        for (int c = 0; c < 7 && ok; ++c) {
            if (!cnt) continue;
            ok = dst[c] ? std::fread(dst[c] + k0, sizeof(double), cnt, f) == cnt
                        : std::fseek(f, (long)(cnt * sizeof(double)), SEEK_CUR) == 0;
        }
    }
    std::fclose(f);
    if (!ok) return RTB_BAD_VALUE;
    if (host_rays->flag)
        for (size_t k = 0; k < hdr[0]; ++k) host_rays->flag[k] = (k < hdr[1]) ? 1 : 0;
    return RTB_OK;
}

int rtb_write_fits(const char* path, const double* image, uint64_t xdim, uint64_t ydim, const char* const* keys,
                   const char* const* values, size_t n_keys) {
    if (!path || !image || xdim == 0 || ydim == 0 || (n_keys && (!keys || !values))) return RTB_BAD_VALUE;
    std::string h;
    h += card("SIMPLE", "T", "file does conform to FITS standard");
    h += card("BITPIX", "-64", "number of bits per data pixel");
    h += card("NAXIS", "2", "number of data axes");
    h += card("NAXIS1", std::to_string(xdim), "length of data axis 1");
    h += card("NAXIS2", std::to_string(ydim), "length of data axis 2");
    h += card("EXTEND", "T", "FITS dataset may contain extensions");
    for (size_t k = 0; k < n_keys; ++k) h += card(keys[k], fits_string(values[k]));
    h += card("END", "");
    h.resize((h.size() + 2879) / 2880 * 2880, ' ');
    FILE* f = std::fopen(path, "wb");
    if (!f) return RTB_FAILED;
    bool ok = put(f, h.data(), h.size());
    std::vector<unsigned char> buf(8 * 4096);
    const uint64_t total = xdim * ydim;
    for (uint64_t i = 0; i < total && ok;) {
        const uint64_t m = (total - i < 4096) ? total - i : 4096;
        for (uint64_t j = 0; j < m; ++j) {
            uint64_t bits;
            std::memcpy(&bits, image + i + j, 8);
            for (int b = 0; b < 8; ++b) buf[8 * j + b] = (unsigned char)(bits >> (56 - 8 * b));  // big-endian
        }
        ok = put(f, buf.data(), 8 * m);
        i += m;
    }
    const size_t data = 8 * total, pad = (data + 2879) / 2880 * 2880 - data;
    std::vector<unsigned char> zeros(pad, 0);
    if (ok) ok = put(f, zeros.data(), pad);
    ok = (std::fclose(f) == 0) && ok;
    return ok ? RTB_OK : RTB_FAILED;
}

}  // extern "C"
