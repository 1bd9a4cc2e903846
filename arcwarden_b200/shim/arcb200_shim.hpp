// arcb200_shim.hpp — glue between the reference's C++ API (namespace arc) and the
// libarcb200 C ABI (include/arcb200.h).
//
// The shim is header-only. Put arcwarden_b200/shim first on the include path and
// the ArcWarden include directory after it:
//
//     nvcc -std=c++20 -I arcwarden_b200/shim -I <ArcWarden>/include tool.cu \
//          -L arcwarden_b200 -larcb200 -lcufft -Xlinker -rpath,<repo>/arcwarden_b200
//
// The shim's pic/*.hpp replace the hot-path headers (particles, depositor,
// pusher, spectral, solver_es, solver_darwin, pump, simulation) and the
// diagnostics (reduced on the GPU, copied back asynchronously) with classes of
// the same names and signatures that call the library; every other pic/*.hpp
// (grid, config, device_array, cuda_utils, species, sources, fields, deck, the
// Yee branch, ...) is the reference's own. Data stays in
// the reference's containers (DeviceArray in Particles, Sources, Fields): the
// library works on those arrays in place, bound by pointer before each call.
//
// Errors: a non-zero status from the library throws arc::CudaError with the
// library's message, as the reference's CUDA_CHECK does.
#ifndef ARC_B200_SHIM_HPP
#define ARC_B200_SHIM_HPP

#include "../../include/arcb200.h"

#include "pic/config.hpp"
#include "pic/cuda_utils.hpp"
#include "pic/fields.hpp"
#include "pic/grid.hpp"
#include "pic/sources.hpp"

#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <tuple>

namespace arc {
namespace shim {

inline void check(int rc, const char* what) {
    if (rc != AW_OK) {
        char buf[1024];
        aw_last_error(buf, sizeof(buf));
        throw CudaError(std::string("libarcb200 ") + what + ": " + buf);
    }
}

// RunParams -> the fields the library reads; has_b0 from SimConfig::has_b0.
inline aw_params params(const RunParams& rp, bool has_b0) {
    aw_params p{};
    p.dt = rp.dt; p.qm = rp.qm; p.eps0 = rp.eps0; p.n0 = rp.n0; p.c = rp.c;
    for (int d = 0; d < 3; ++d) p.B0[d] = rp.B0[d];
    p.has_b0 = has_b0 ? 1 : 0;
    p.pump = rp.pump ? 1 : 0;
    p.pump_ex = rp.pump_ex; p.pump_ey = rp.pump_ey; p.pump_ez = rp.pump_ez;
    p.pump_k0 = rp.pump_k0; p.pump_w0 = rp.pump_w0;
    p.pump_trmp = rp.pump_trmp; p.pump_toff = rp.pump_toff;
    return p;
}

inline aw_grid grid_of(const Grid& g) { return aw_grid{g.nx, g.ny, g.Lx, g.Ly}; }

// One library context per (grid, field model) for the stand-alone operators
// (Depositor, Pusher, the solvers, SpectralEngine, Particles). Contexts live
// until the process exits; the simulation class owns its own.
inline aw_ctx* context(const Grid& g, int model) {
    static std::mutex mu;
    static std::map<std::tuple<int, int, double, double, int>, aw_ctx*> cache;
    std::lock_guard<std::mutex> lock(mu);
    const auto key = std::make_tuple(g.nx, g.ny, g.Lx, g.Ly, model);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    const aw_grid ag = grid_of(g);
    const aw_params ap = params(RunParams{}, true);
    aw_ctx* c = nullptr;
    check(aw_ctx_create(&ag, &ap, model, nullptr, &c), "context");
    cache.emplace(key, c);
    return c;
}

// The grid of the most recent call on this thread (for calls that name none).
inline Grid& last_grid() {
    thread_local Grid g;
    return g;
}

// A context prepared for one call: stream and parameters set.
inline aw_ctx* prepare(const Grid& g, const RunParams& rp, bool has_b0, cudaStream_t s,
                       int model = AW_MODEL_DARWIN) {
    last_grid() = g;
    aw_ctx* c = context(g, model);
    check(aw_set_stream(c, s), "set_stream");
    const aw_params p = params(rp, has_b0);
    check(aw_set_params(c, &p), "set_params");
    return c;
}

inline aw_source_ptrs source_ptrs(Sources& s) {
    return aw_source_ptrs{s.rho.data(), s.Jx.data(), s.Jy.data(), s.Jz.data(), s.dcux.data(), s.dcuy.data(),
                          s.dcuz.data(), s.amu0.data(), s.amu1.data(), s.amu2.data(), s.amu3.data()};
}
inline aw_field_ptrs field_ptrs(Fields& f) {
    return aw_field_ptrs{f.Ex.data(), f.Ey.data(), f.Ez.data(), f.Bx.data(), f.By.data(), f.Bz.data(),
                         f.ELx.data(), f.ELy.data(), f.ETx.data(), f.ETy.data(), f.ETz.data()};
}
inline void bind_sources(aw_ctx* c, Sources& s) {
    const aw_source_ptrs p = source_ptrs(s);
    check(aw_sources_bind(c, &p), "sources_bind");
}
inline void bind_fields(aw_ctx* c, Fields& f) {
    const aw_field_ptrs p = field_ptrs(f);
    check(aw_fields_bind(c, &p), "fields_bind");
}

}  // namespace shim
}  // namespace arc

#endif  // ARC_B200_SHIM_HPP
