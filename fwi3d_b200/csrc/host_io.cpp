// host_io.cpp -- the reference's host-side file formats behind the C ABI:
// parameters.txt lookup, SPS/RPS point files and raw float32 binaries.
// Host code only (no device work); compiled into libfwi3d.so.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/fwi3d.h"

namespace {

int copy_out(const std::string &v, char *out, int cap)
{
    if (!out || cap <= 0) return FWI_ERR_ARG;
    if ((int)v.size() >= cap) return FWI_ERR_ARG;
    memcpy(out, v.c_str(), v.size() + 1);
    return FWI_OK;
}

}  // namespace

extern "C" {

// catch_parameter (src/admin/admin.cpp:53-88): the first line that does not
// start with '#' or ' ' and starts with `key` (a prefix match) gives the
// value: the text from two characters after the first '=' up to a '#', with
// every space removed.  A missing key gives an empty value (FWI_OK), an
// unreadable file FWI_ERR_IO.
int fwi_catch_parameter(const char *file, const char *key, char *value, int cap)
{
    if (!file || !key) return FWI_ERR_ARG;
    std::ifstream in(file);
    if (!in.is_open()) return FWI_ERR_IO;
    std::string line, v;
    const std::string target(key);
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '#' || line[0] == ' ') continue;
        if (line.compare(0, target.size(), target) != 0) continue;
        // find("=") + 2 wraps to 1 when there is no '=' (size_t arithmetic)
        const size_t eq = line.find('=');
        for (size_t i = eq + 2; i < line.size(); ++i) {
            if (line[i] == '#') break;
            v += line[i];
        }
        break;
    }
    v.erase(std::remove(v.begin(), v.end(), ' '), v.end());
    return copy_out(v, value, cap);
}

// SPS/RPS point file (src/geometry/geometry.cpp:3-47 with import_text_file,
// src/admin/admin.cpp:39-51): one "x,y,z" line per point in metres, lines
// starting with '#' skipped.  With x == NULL only the count is returned.
int fwi_read_points(const char *file, float *x, float *y, float *z, int cap, int *n)
{
    if (!file || !n) return FWI_ERR_ARG;
    std::ifstream in(file);
    if (!in.is_open()) return FWI_ERR_IO;
    std::string line;
    int k = 0;
    while (std::getline(in, line)) {
        if (!line.empty() && line[0] == '#') continue;
        if (line.empty()) continue;
        if (x) {
            if (k >= cap) return FWI_ERR_ARG;
            std::stringstream ss(line);
            std::string tok[3];
            for (int a = 0; a < 3; ++a)
                if (!std::getline(ss, tok[a], ',')) return FWI_ERR_ARG;
            try {
                x[k] = std::stof(tok[0]);
                y[k] = std::stof(tok[1]);
                z[k] = std::stof(tok[2]);
            } catch (...) {
                return FWI_ERR_ARG;
            }
        }
        ++k;
    }
    *n = k;
    return FWI_OK;
}

// import_binary_float / export_binary_float (src/admin/admin.cpp:13-37).
int fwi_read_binary(const char *file, float *buf, int64_t n)
{
    if (!file || (!buf && n > 0) || n < 0) return FWI_ERR_ARG;
    FILE *f = fopen(file, "rb");
    if (!f) return FWI_ERR_IO;
    const size_t got = fread(buf, sizeof(float), (size_t)n, f);
    fclose(f);
    return got == (size_t)n ? FWI_OK : FWI_ERR_IO;
}

int fwi_write_binary(const char *file, const float *buf, int64_t n)
{
    if (!file || (!buf && n > 0) || n < 0) return FWI_ERR_ARG;
    FILE *f = fopen(file, "wb");
    if (!f) return FWI_ERR_IO;
    const size_t put = fwrite(buf, sizeof(float), (size_t)n, f);
    fclose(f);
    return put == (size_t)n ? FWI_OK : FWI_ERR_IO;
}

}  // extern "C"
