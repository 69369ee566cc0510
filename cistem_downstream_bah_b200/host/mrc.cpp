// mrc.cpp -- MRC2014 reading and writing (see mrc.hpp).
#include "mrc.hpp"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>

namespace tmhost {

namespace {
struct Header {
    int32_t nx, ny, nz, mode, nxstart, nystart, nzstart, mx, my, mz;
    float cella[3], cellb[3];
    int32_t mapc, mapr, maps;
    float dmin, dmax, dmean;
    int32_t ispg, nsymbt;
    int32_t extra[25];
    float origin[3];
    char map[4];
    unsigned char machst[4];
    float rms;
    int32_t nlabl;
    char labels[10][80];
};
static_assert(sizeof(Header) == 1024, "MRC header is 1024 bytes");
}  // namespace

bool read_mrc(const std::string& path, MrcData& out, std::string& err, int first_slice, int last_slice) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) { err = "cannot open " + path; return false; }
    Header h;
    if (std::fread(&h, sizeof h, 1, f) != 1) { std::fclose(f); err = "short MRC header in " + path; return false; }
    if (h.nx <= 0 || h.ny <= 0 || h.nz <= 0) { std::fclose(f); err = "bad MRC dimensions in " + path; return false; }
    int bytes;
    switch (h.mode) {
        case 0: bytes = 1; break;
        case 1: case 6: case 12: bytes = 2; break;
        case 2: bytes = 4; break;
        default: std::fclose(f); err = "unsupported MRC mode " + std::to_string(h.mode) + " in " + path; return false;
    }
    if (last_slice <= 0) last_slice = h.nz;
    if (first_slice < 1 || last_slice > h.nz || first_slice > last_slice) {
        std::fclose(f);
        err = "slice range outside the file " + path;
        return false;
    }
    const size_t slice = (size_t)h.nx * h.ny;
    const int nz = last_slice - first_slice + 1;
    if (std::fseek(f, 1024L + h.nsymbt + (long)((first_slice - 1) * slice * bytes), SEEK_SET) != 0) {
        std::fclose(f);
        err = "seek failed in " + path;
        return false;
    }
    std::vector<unsigned char> raw(slice * nz * bytes);
    if (std::fread(raw.data(), 1, raw.size(), f) != raw.size()) {
        std::fclose(f);
        err = "truncated MRC data in " + path;
        return false;
    }
    std::fclose(f);
    out.nx = h.nx;
    out.ny = h.ny;
    out.nz = nz;
    out.pixel_size = (h.cella[0] != 0.f && h.mx > 0) ? h.cella[0] / (float)h.mx : 0.f;
    out.data.resize(slice * nz);
    for (size_t i = 0; i < out.data.size(); i++) {
        switch (h.mode) {
            case 0: out.data[i] = (float)(int8_t)raw[i]; break;
            case 1: { int16_t v; std::memcpy(&v, &raw[2 * i], 2); out.data[i] = v; break; }
            case 6: { uint16_t v; std::memcpy(&v, &raw[2 * i], 2); out.data[i] = v; break; }
            case 12: {
                uint16_t v;
                std::memcpy(&v, &raw[2 * i], 2);
                // IEEE half to float
                const uint32_t sign = (v & 0x8000u) << 16, e = (v >> 10) & 0x1f, m = v & 0x3ff;
                float val;
                if (e == 0) val = std::ldexp((float)m, -24);
                else if (e == 31) val = m ? NAN : INFINITY;
                else val = std::ldexp((float)(m | 0x400), (int)e - 25);
                out.data[i] = sign ? -val : val;
                break;
            }
            default: { float v; std::memcpy(&v, &raw[4 * i], 4); out.data[i] = v; }
        }
    }
    return true;
}

bool write_mrc(const std::string& path, int nx, int ny, int nz, const float* data, float pixel_size, std::string& err) {
    Header h;
    std::memset(&h, 0, sizeof h);
    h.nx = h.mx = nx;
    h.ny = h.my = ny;
    h.nz = h.mz = nz;
    h.mode = 2;
    h.cella[0] = pixel_size * nx;
    h.cella[1] = pixel_size * ny;
    h.cella[2] = pixel_size * nz;
    h.cellb[0] = h.cellb[1] = h.cellb[2] = 90.f;
    h.mapc = 1; h.mapr = 2; h.maps = 3;
    h.ispg = 1;
    const size_t n = (size_t)nx * ny * nz;
    double sum = 0, sum2 = 0;
    float mn = n ? data[0] : 0.f, mx = n ? data[0] : 0.f;
    for (size_t i = 0; i < n; i++) {
        sum += data[i];
        sum2 += (double)data[i] * data[i];
        if (data[i] < mn) mn = data[i];
        if (data[i] > mx) mx = data[i];
    }
    h.dmin = mn;
    h.dmax = mx;
    h.dmean = n ? (float)(sum / n) : 0.f;
    h.rms = n ? (float)std::sqrt(std::fmax(0.0, sum2 / n - (sum / n) * (sum / n))) : 0.f;
    std::memcpy(h.map, "MAP ", 4);
    h.machst[0] = 0x44; h.machst[1] = 0x44;
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) { err = "cannot write " + path; return false; }
    bool ok = std::fwrite(&h, sizeof h, 1, f) == 1 && std::fwrite(data, sizeof(float), n, f) == n;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) err = "write failed for " + path;
    return ok;
}

}  // namespace tmhost
