// pic/particles.hpp (B200 shim) — the reference's Particles container
// (include/pic/particles.hpp:453-727) with its loader, migrate and tile binning
// done by libarcb200. The data members, the view structs and the method
// signatures are the reference's, so code written against it (the tools, the
// tests, the diagnostics and the Yee branch) compiles unchanged.
#ifndef ARC_PIC_PARTICLES_HPP
#define ARC_PIC_PARTICLES_HPP

#include "pic/config.hpp"
#include "pic/cuda_utils.hpp"
#include "pic/device_array.hpp"
#include "pic/grid.hpp"
#include "pic/species.hpp"

#include "../arcb200_shim.hpp"

#include <cstddef>
#include <stdexcept>
#include <vector>

namespace arc {

// Device views of the particle SoA (same members as the reference's).
struct ParticleViews {
    DeviceView<float> x, y, ux, uy, uz;
    DeviceView<float> w;
    DeviceView<float> wd;
    DeviceView<int>   cell;
    int n = 0;
    DeviceView<float>  wc;
    DeviceView<double> wdd;
};

// Tile binning: tile t owns idx[off[t] .. off[t+1]) (idx empty after a
// physical sort, when the particles themselves are in tile order).
struct BinViews {
    DeviceView<int> off;
    DeviceView<int> idx;
    int ntiles = 0;
    int ntx = 0;
    int tx = 0, ty = 0;
};

namespace detail {
__host__ __device__ inline int tile_of(int cell, int nx, int tx, int ty, int ntx) {
    return ((cell / nx) / ty) * ntx + (cell % nx) / tx;
}
}  // namespace detail

struct Particles {
    DeviceArray<float> x, y;
    DeviceArray<float> ux, uy, uz;
    DeviceArray<float> w;
    DeviceArray<int>   cell;
    std::size_t        n = 0;

    DeviceArray<int> bin_count, bin_off, bin_cursor, bin_idx;
    int bin_ntiles = 0, bin_ntx = 0, bin_tx = 0, bin_ty = 0;
    bool sorted = false;

    DeviceArray<float> x2, y2, ux2, uy2, uz2, w2;
    DeviceArray<int>   cell2;

    DeviceArray<float> wd, wd2;
    bool has_wd = false;
    DeviceArray<float>  wc;
    DeviceArray<double> wdd;
    int wprec = 0;

    // The stream the particles were last loaded on (an addition to the
    // reference's members): the deck diagnostics enqueue their device work on
    // it. nullptr = the legacy default stream.
    cudaStream_t stream = nullptr;

    Particles() = default;

    void enable_deltaf(cudaStream_t s, int wprec_ = 0) {
        wd = DeviceArray<float>(n);
        wd.zero(s);
        has_wd = true;
        wprec = wprec_;
        if (wprec == 1) { wc = DeviceArray<float>(n); wc.zero(s); }
        if (wprec == 2) { wdd = DeviceArray<double>(n); wdd.zero(s); }
    }

    void allocate_n(std::size_t n_total) {
        n = n_total;
        x = DeviceArray<float>(n); y = DeviceArray<float>(n);
        ux = DeviceArray<float>(n); uy = DeviceArray<float>(n); uz = DeviceArray<float>(n);
        w = DeviceArray<float>(n);
        cell = DeviceArray<int>(n);
    }
    void allocate(const Grid& g, int ppc) {
        allocate_n(static_cast<std::size_t>(g.real_size()) * static_cast<std::size_t>(ppc));
    }

    ParticleViews views() {
        return ParticleViews{x.view(), y.view(), ux.view(), uy.view(), uz.view(), w.view(), wd.view(),
                             cell.view(), static_cast<int>(n), wc.view(), wdd.view()};
    }
    BinViews bins() {
        return BinViews{bin_off.view(), bin_idx.view(), bin_ntiles, bin_ntx, bin_tx, bin_ty};
    }

    // Bind this container to a library context (on the context's stream).
    void bind(aw_ctx* c) {
        shim::check(aw_particles_bind(c, x.data(), y.data(), ux.data(), uy.data(), uz.data(), w.data(),
                                      cell.data(), static_cast<int64_t>(n)),
                    "particles_bind");
    }

    // Single-species RunParams load (aw_load_legacy).
    void initialize(const RunParams& rp, const Grid& g, cudaStream_t s) {
        if (n == 0) allocate(g, rp.ppc);
        stream = s;
        aw_ctx* c = shim::prepare(g, rp, true, s);
        bind(c);
        aw_legacy_load L{};
        L.ppc = rp.ppc; L.weight = rp.weight; L.vth = rp.vth; L.vd = rp.vd;
        L.two_stream = rp.two_stream ? 1 : 0; L.bump_on_tail = rp.bump_on_tail ? 1 : 0;
        L.beam_frac = rp.beam_frac; L.beam_vd = rp.beam_vd; L.beam_vth = rp.beam_vth;
        L.perturb_amp = rp.perturb_amp; L.perturb_kx = rp.perturb_kx;
        L.noisy = rp.noisy_load ? 1 : 0;
        L.seed = static_cast<uint64_t>(rp.rng_seed);
        shim::check(aw_load_legacy(c, &L), "load_legacy");
        sorted = false;
    }

    // Multi-species load (aw_load_species): species k fills its own slice.
    void initialize(const SpeciesList& sp, const Grid& g, const RunParams& rp, cudaStream_t s) {
        std::size_t total = 0;
        for (const auto& q : sp) total += static_cast<std::size_t>(q.ppc) * g.real_size();
        if (total == 0) return;
        allocate_n(total);
        stream = s;
        std::vector<aw_species> a;
        for (const auto& q : sp) {
            aw_species e{};
            e.ppc = q.ppc; e.density = q.density;
            for (int d = 0; d < 3; ++d) { e.uth[d] = q.uth[d]; e.ufl[d] = q.ufl[d]; }
            a.push_back(e);
        }
        aw_ctx* c = shim::prepare(g, rp, true, s);
        bind(c);
        shim::check(aw_load_species(c, a.data(), static_cast<int32_t>(a.size()),
                                    static_cast<uint64_t>(rp.rng_seed), rp.noisy_load ? 1 : 0),
                    "load_species");
        sorted = false;
    }

    // Mirror-geometry loads belong to the 1D hybrid code, outside this library.
    void initialize_mirror(const Species&, const Grid&, const RunParams&, cudaStream_t) {
        throw std::runtime_error("Particles::initialize_mirror is not provided by the B200 library");
    }

    void migrate(const Grid& g, cudaStream_t s) {
        aw_ctx* c = shim::prepare(g, RunParams{}, true, s);
        bind(c);
        shim::check(aw_migrate(c), "migrate");
    }

    void build_tile_bins(const Grid& g, int tx, int ty, cudaStream_t s) { tile_bins(g, tx, ty, s, false); }
    void sort_by_tile(const Grid& g, int tx, int ty, cudaStream_t s) { tile_bins(g, tx, ty, s, true); }

private:
    void tile_bins(const Grid& g, int tx, int ty, cudaStream_t s, bool physical) {
        aw_ctx* c = shim::prepare(g, RunParams{}, true, s);
        bind(c);
        shim::check(aw_sort_tiles(c, tx, ty, physical ? 1 : 0), "sort_tiles");
        const int32_t* off = nullptr;
        const int32_t* idx = nullptr;
        int32_t ntiles = 0, ntx = 0;
        shim::check(aw_tile_bins(c, &off, &idx, &ntiles, &ntx), "tile_bins");
        if (bin_off.size() != static_cast<std::size_t>(ntiles) + 1)
            bin_off = DeviceArray<int>(static_cast<std::size_t>(ntiles) + 1);
        CUDA_CHECK(cudaMemcpyAsync(bin_off.data(), off, sizeof(int) * (ntiles + 1), cudaMemcpyDeviceToDevice, s));
        if (!physical) {
            if (bin_idx.size() != n) bin_idx = DeviceArray<int>(n);
            CUDA_CHECK(cudaMemcpyAsync(bin_idx.data(), idx, sizeof(int) * n, cudaMemcpyDeviceToDevice, s));
        }
        bin_ntiles = ntiles; bin_ntx = ntx; bin_tx = tx; bin_ty = ty;
        sorted = physical;
    }
};

}  // namespace arc

#endif  // ARC_PIC_PARTICLES_HPP
