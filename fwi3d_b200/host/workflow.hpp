// workflow.hpp -- host side of the drop-in executables: the reference's
// parameters.txt keys, SPS/RPS geometry and raw binary layouts over the C ABI.
#pragma once

#include <chrono>
#include <cmath>
#include <cstdio>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "fwi3d.h"

namespace fwh {

// A failing ABI call becomes an exception with the library's message; main()
// prints it in red and exits 1, like the reference's uncaught
// std::invalid_argument (src/admin/admin.cpp:17-18).
inline void check(int st, fwi_ctx *ctx, const char *what)
{
    if (st == FWI_OK) return;
    std::string msg = std::string(what) + ": " + fwi_status_string(st);
    if (ctx) {
        char buf[512] = {0};
        fwi_last_error(ctx, buf, sizeof buf);
        if (buf[0]) msg += std::string(" (") + buf + ")";
    }
    throw std::runtime_error(msg);
}

// catch_parameter(key, file) (src/admin/admin.cpp:53-88).
inline std::string param(const std::string &file, const std::string &key)
{
    char buf[4096];
    const int st = fwi_catch_parameter(file.c_str(), key.c_str(), buf, sizeof buf);
    if (st == FWI_ERR_IO) throw std::invalid_argument("Error: \033[31m" + file + "\033[0;0m could not be opened!");
    check(st, nullptr, ("parameter " + key).c_str());
    return std::string(buf);
}

inline int param_i(const std::string &file, const std::string &key) { return std::stoi(param(file, key)); }
inline float param_f(const std::string &file, const std::string &key) { return std::stof(param(file, key)); }

// Optional project keys (prefix "b200_", which no reference key starts with).
inline int opt_i(const std::string &file, const std::string &key, int dflt)
{
    const std::string v = param(file, key);
    return v.empty() ? dflt : std::stoi(v);
}

struct Points {
    std::vector<float> x, y, z;
    int n = 0;
};

inline Points read_points(const std::string &file)
{
    Points p;
    int n = 0;
    int st = fwi_read_points(file.c_str(), nullptr, nullptr, nullptr, 0, &n);
    if (st == FWI_ERR_IO) throw std::invalid_argument("Error: \033[31m" + file + "\033[0;0m could not be opened!");
    check(st, nullptr, file.c_str());
    p.x.resize(n);
    p.y.resize(n);
    p.z.resize(n);
    check(fwi_read_points(file.c_str(), p.x.data(), p.y.data(), p.z.data(), n, &n), nullptr, file.c_str());
    p.n = n;
    return p;
}

inline void read_binary(const std::string &file, float *buf, size_t n)
{
    const int st = fwi_read_binary(file.c_str(), buf, (int64_t)n);
    if (st == FWI_ERR_IO) throw std::invalid_argument("Error: \033[31m" + file + "\033[0;0m could not be opened!");
    check(st, nullptr, file.c_str());
}

inline void write_binary(const std::string &file, const float *buf, size_t n)
{
    const int st = fwi_write_binary(file.c_str(), buf, (int64_t)n);
    if (st == FWI_ERR_IO) throw std::invalid_argument("Error: \033[31m" + file + "\033[0;0m could not be opened!");
    check(st, nullptr, file.c_str());
    std::cout << "\nBinary file \033[34m" << file << "\033[0;0m was successfully written." << std::endl;
}

// The model block every main reads (src/modeling/modeling.cu:17-34).
struct Model {
    int nx, ny, nz, nt;
    float dh, dt, fmax;
    std::vector<float> vp;  // [nz,nx,ny], z fastest
    Points src, rec;
};

inline Model read_model(const std::string &pf)
{
    Model m;
    m.nx = param_i(pf, "x_samples");
    m.ny = param_i(pf, "y_samples");
    m.nz = param_i(pf, "z_samples");
    m.dh = param_f(pf, "model_spacing");
    m.nt = param_i(pf, "time_samples");
    m.dt = param_f(pf, "time_spacing");
    m.fmax = param_f(pf, "max_frequency");
    m.vp.resize((size_t)m.nx * m.ny * m.nz);
    read_binary(param(pf, "model_file"), m.vp.data(), m.vp.size());
    m.src = read_points(param(pf, "SPS"));
    m.rec = read_points(param(pf, "RPS"));
    return m;
}

// Pad width: int(length / dh) + 1 (src/modeling/modeling.cu:90, migration.cu:13).
inline int pad_cells(float length, float dh) { return (int)(length / dh) + 1; }

inline fwi_ctx *make_context(const Model &m, int nb, int boundary, float abc_factor, int batch, int flags)
{
    fwi_grid g{m.nz, m.nx, m.ny, nb, m.dh};
    fwi_params p{m.nt, m.dt, m.fmax, boundary, abc_factor, batch, flags};
    fwi_ctx *ctx = nullptr;
    check(fwi_create(&g, &p, &ctx), nullptr, "fwi_create");
    check(fwi_set_geometry(ctx, m.src.n, m.src.x.data(), m.src.y.data(), m.src.z.data(), m.rec.n, m.rec.x.data(),
                           m.rec.y.data(), m.rec.z.data(), nullptr, nullptr),
          ctx, "fwi_set_geometry");
    return ctx;
}

struct Clock {
    std::chrono::system_clock::time_point t0 = std::chrono::system_clock::now();
    double seconds() const
    {
        return std::chrono::duration<double>(std::chrono::system_clock::now() - t0).count();
    }
};

inline std::string banner(const std::string &title)
{
    const std::string line(80, '-');
    return line + "\n" + std::string((80 - (int)title.size()) / 2, ' ') + title + "\n" + line + "\n";
}

}  // namespace fwh
