// pic/depositor.hpp (B200 shim) — Depositor<Cfg> (include/pic/depositor.hpp:
// 326-497) on libarcb200. Every policy (global, shared-tile, tiled) computes the
// same exact fixed-point deposit, so the Cfg's deposit tag selects nothing;
// as in the reference, the deposits ADD into the sources and the caller zeroes
// them. charge_current_sorted first sorts the particles physically by 16x16
// tile, like the reference.
#ifndef ARC_PIC_DEPOSITOR_HPP
#define ARC_PIC_DEPOSITOR_HPP

#include "pic/config.hpp"
#include "pic/cuda_utils.hpp"
#include "pic/fields.hpp"
#include "pic/grid.hpp"
#include "pic/particles.hpp"
#include "pic/sources.hpp"

#include "../arcb200_shim.hpp"
#include "../../csrc/aw_device.cuh"

namespace arc {

// Per-particle CIC charge deposit over the given views (the reference's
// kernel-level entry, depositor.hpp:35-58; its tests launch it directly to
// check the CIC arithmetic): rho += coef * w_k with FP32 global atomics, any
// launch shape (grid-stride loop). The weights and coef are the library's.
template <class Cfg, class Policy = AtomicGlobalDeposit>
__global__ void deposit_charge_kernel(ParticleViews p, SourceViews s, Grid g, RunParams rp) {
    const double qoa = rp.qm / (g.dx * g.dy);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < p.n; t += gridDim.x * blockDim.x) {
        const float x = p.x[t], y = p.y[t];
        if (!(x >= 0.0f && x < static_cast<float>(g.nx) && y >= 0.0f && y < static_cast<float>(g.ny))) continue;
        const aw::Cic c = aw::cic(x, y);
        const int i1 = aw::wrap_once(c.i0 + 1, g.nx), j1 = aw::wrap_once(c.j0 + 1, g.ny);
        const float coef = __double2float_rn(qoa * static_cast<double>(p.w[t]));
        atomicAdd(&s.rho[c.j0 * g.nx + c.i0], coef * c.w0);
        atomicAdd(&s.rho[c.j0 * g.nx + i1], coef * c.w1);
        atomicAdd(&s.rho[j1 * g.nx + c.i0], coef * c.w2);
        atomicAdd(&s.rho[j1 * g.nx + i1], coef * c.w3);
    }
}

template <class Cfg>
struct Depositor {
    static constexpr int kThreads = 256;

    static void charge(Particles& parts, Sources& src, const Grid& g, const RunParams& rp, cudaStream_t s) {
        run(parts, src, nullptr, g, rp, s, aw_deposit_rho, "deposit_rho");
    }
    static void charge_tiled(Particles& parts, Sources& src, const Grid& g, const RunParams& rp,
                             cudaStream_t s) {
        charge(parts, src, g, rp, s);
    }
    static void charge_current(Particles& parts, Sources& src, const Grid& g, const RunParams& rp,
                               cudaStream_t s) {
        run(parts, src, nullptr, g, rp, s, aw_deposit_rho_j, "deposit_rho_j");
    }
    static void charge_current_sorted(Particles& parts, Sources& src, const Grid& g, const RunParams& rp,
                                      cudaStream_t s) {
        parts.sort_by_tile(g, 16, 16, s);
        charge_current(parts, src, g, rp, s);
    }
    static void deposit_amu(Particles& parts, Sources& src, const Grid& g, const RunParams& rp,
                            cudaStream_t s) {
        run(parts, src, nullptr, g, rp, s, aw_deposit_amu, "deposit_amu");
    }
    static void deposit_dcu(Particles& parts, Sources& src, const Fields& flds, const Grid& g,
                            const RunParams& rp, cudaStream_t s) {
        run(parts, src, &flds, g, rp, s, aw_deposit_dcu, "deposit_dcu");
    }

private:
    static void run(Particles& parts, Sources& src, const Fields* flds, const Grid& g, const RunParams& rp,
                    cudaStream_t s, int (*op)(aw_ctx*), const char* what) {
        aw_ctx* c = shim::prepare(g, rp, Cfg::has_b0, s);
        parts.bind(c);
        shim::bind_sources(c, src);
        if (flds) shim::bind_fields(c, const_cast<Fields&>(*flds));
        shim::check(op(c), what);
    }
};

}  // namespace arc

#endif  // ARC_PIC_DEPOSITOR_HPP
