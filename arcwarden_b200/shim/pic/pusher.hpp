// pic/pusher.hpp (B200 shim) — Pusher<Cfg> (include/pic/pusher.hpp:262-331) on
// libarcb200, plus the device Boris rotation other headers call
// (detail::boris_rotate, pusher.hpp:85-97; the Yee branch uses it).
#ifndef ARC_PIC_PUSHER_HPP
#define ARC_PIC_PUSHER_HPP

#include "pic/config.hpp"
#include "pic/cuda_utils.hpp"
#include "pic/fields.hpp"
#include "pic/grid.hpp"
#include "pic/particles.hpp"

#include "../arcb200_shim.hpp"
#include "../../csrc/aw_device.cuh"

namespace arc {
namespace detail {

// Rotation of u about B with qmh = (q/m) dt/2 (the library's own Boris step).
__device__ inline void boris_rotate(float& ux, float& uy, float& uz, float Bx, float By, float Bz, float qmh) {
    aw::boris_rotate(ux, uy, uz, Bx, By, Bz, qmh);
}

// One-thread-per-particle ES push over the given views (the reference's
// kernel-level entry, pusher.hpp:113-129; its tests launch it directly): CIC
// gather of Ex, Ey, Boris about rp.B0 when Cfg::has_b0, move without wrap.
// The arithmetic is the library's own (aw_device.cuh).
template <class Cfg>
__global__ void boris_push_kernel(ParticleViews p, FieldViews f, Grid g, RunParams rp) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= p.n) return;
    const float x = p.x[t], y = p.y[t];
    const aw::Cic c = aw::cic(x, y);
    const int i1 = aw::wrap_once(c.i0 + 1, g.nx), j1 = aw::wrap_once(c.j0 + 1, g.ny);
    const int c0 = c.j0 * g.nx + c.i0, c1 = c.j0 * g.nx + i1, c2 = j1 * g.nx + c.i0, c3 = j1 * g.nx + i1;
    const float ex = aw::gather4(c, f.Ex[c0], f.Ex[c1], f.Ex[c2], f.Ex[c3]);
    const float ey = aw::gather4(c, f.Ey[c0], f.Ey[c1], f.Ey[c2], f.Ey[c3]);
    float ux = p.ux[t], uy = p.uy[t], uz = p.uz[t];
    const float qmh = static_cast<float>(rp.qm) * 0.5f * static_cast<float>(rp.dt);
    aw::boris_es(ux, uy, uz, ex, ey, qmh, Cfg::has_b0, rp.B0[0], rp.B0[1], rp.B0[2]);
    p.ux[t] = ux; p.uy[t] = uy; p.uz[t] = uz;
    p.x[t] = aw::move1(x, ux, rp.dt, g.dx);
    p.y[t] = aw::move1(y, uy, rp.dt, g.dy);
}

}  // namespace detail

template <class Cfg>
struct Pusher {
    // ES push (gather Ex, Ey; Boris about rp.B0 when Cfg::has_b0; move).
    static void boris(Particles& parts, const Fields& flds, const Grid& g, const RunParams& rp, cudaStream_t s) {
        run(parts, flds, g, rp, s, aw_push_es, "push_es");
    }
    static void boris_tiled(Particles& parts, const Fields& flds, const Grid& g, const RunParams& rp,
                            cudaStream_t s) {
        boris(parts, flds, g, rp, s);
    }
    // EM push (gather E_total and B; full Boris; move).
    static void boris_em(Particles& parts, const Fields& flds, const Grid& g, const RunParams& rp,
                         cudaStream_t s) {
        run(parts, flds, g, rp, s, aw_push_em, "push_em");
    }
    // u(t) -> u(t - dt/2) from the current E (no move).
    static void half_step_back(Particles& parts, const Fields& flds, const Grid& g, const RunParams& rp,
                               cudaStream_t s) {
        run(parts, flds, g, rp, s, aw_half_step_back, "half_step_back");
    }

private:
    static void run(Particles& parts, const Fields& flds, const Grid& g, const RunParams& rp, cudaStream_t s,
                    int (*op)(aw_ctx*), const char* what) {
        aw_ctx* c = shim::prepare(g, rp, Cfg::has_b0, s);
        parts.bind(c);
        shim::bind_fields(c, const_cast<Fields&>(flds));
        shim::check(op(c), what);
    }
};

}  // namespace arc

#endif  // ARC_PIC_PUSHER_HPP
