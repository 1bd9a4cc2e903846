// pic/simulation_maxwell.hpp (B200 shim) — MaxwellSimulation
// (include/pic/simulation_maxwell.hpp:25-227) on libarcb200's Yee model
// (AW_MODEL_YEE). The fields stay the reference's YeeFields (its ex_ .. bz_
// and jx_ .. jz_ arrays, bound to the library as fields and sources), the
// particles the shim's Particles. step() is one replay of the library's
// captured Yee step; field_energy() and residuals() are the reference's own
// diagnostics, launched from its header (yee2d.hpp: k_energy, k_rho_nodes,
// k_binomial3x3, k_gauss_residual, k_div_stats).
//
// The library's Yee model is the periodic set: options it does not have
// (relativistic push, delta-f weights, the mirror profile, absorbing layers,
// antenna, cold fluid, more than 4 filter passes) make step() throw. The
// particle order follows the reference's paths: kept on the flat path
// (tile_sort = 0), re-sorted by tile every tile_sort steps otherwise. With no
// particles (a vacuum run) the step is the field half alone.
#ifndef ARC_PIC_SIMULATION_MAXWELL_HPP
#define ARC_PIC_SIMULATION_MAXWELL_HPP

#include "pic/yee2d.hpp"

#include "../arcb200_shim.hpp"

#include <cmath>
#include <stdexcept>

namespace arc {

class MaxwellSimulation {
public:
    MaxwellSimulation(const Grid& g, const RunParams& rp)
        : g_(g), rp_(rp), flds_(g, rp.c, rp.dt), diag_(2), jtmp_(rp.jfilter > 0 ? g.real_size() : 0) {}
    ~MaxwellSimulation() {
        if (ctx_) aw_ctx_destroy(ctx_);
    }
    MaxwellSimulation(const MaxwellSimulation&) = delete;
    MaxwellSimulation& operator=(const MaxwellSimulation&) = delete;

    Grid&       grid()      { return g_; }
    RunParams&  params()    { return rp_; }
    Particles&  particles() { return parts_; }
    YeeFields&  fields()    { return flds_; }
    CudaStream& stream()    { return s_; }
    DeviceArray<float>& vcy() { return vcy_; }
    DeviceArray<float>& vcz() { return vcz_; }

    void step() { step_at(nstep_ * rp_.dt); ++nstep_; }

    void step_at(double tnow) {
        if (rp_.rel || rp_.deltaf || rp_.b0_prof || rp_.bnd_x || rp_.ant_amp != 0.0 || rp_.cold_nc > 0.0 ||
            rp_.jfilter > 4)
            throw CudaError("MaxwellSimulation: this option set is not provided by the B200 library "
                            "(periodic, non-relativistic, uniform B0, jfilter <= 4)");
        if (!ctx_) {
            const aw_grid ag = shim::grid_of(g_);
            const aw_params ap = shim::params(rp_, true);
            shim::check(aw_ctx_create(&ag, &ap, AW_MODEL_YEE, s_.get(), &ctx_), "ctx_create (Yee)");
            shim::check(aw_set_resort(ctx_, rp_.tile_sort > 0 ? rp_.tile_sort : 0), "set_resort");
            shim::check(aw_set_current_filter(ctx_, rp_.jfilter), "set_current_filter");
        }
        parts_.bind(ctx_);
        aw_field_ptrs f{};
        f.Ex = flds_.ex_.data(); f.Ey = flds_.ey_.data(); f.Ez = flds_.ez_.data();
        f.Bx = flds_.bx_.data(); f.By = flds_.by_.data(); f.Bz = flds_.bz_.data();
        shim::check(aw_fields_bind(ctx_, &f), "fields_bind");
        aw_source_ptrs j{};
        j.Jx = flds_.jx_.data(); j.Jy = flds_.jy_.data(); j.Jz = flds_.jz_.data();
        shim::check(aw_sources_bind(ctx_, &j), "sources_bind");
        if (!inited_) {
            shim::check(aw_init(ctx_), "init");
            inited_ = true;
        }
        const long n = std::lround(tnow / rp_.dt);
        shim::check(aw_run(ctx_, n, 1, 1), "run");
    }

    struct Energies { double we, wb; };
    // The reference's k_energy over the current fields.
    Energies field_energy() {
        CUDA_CHECK(cudaMemsetAsync(diag_.data(), 0, diag_.bytes(), s_));
        const int n = g_.real_size();
        yee::k_energy<<<(n + 255) / 256, 256, 0, s_>>>(flds_.views(), diag_.data());
        CUDA_CHECK(cudaPeekAtLastError());
        double h[2];
        CUDA_CHECK(cudaMemcpyAsync(h, diag_.data(), sizeof(h), cudaMemcpyDeviceToHost, s_));
        s_.synchronize();
        return {h[0], h[1]};
    }

    struct Residuals { double divb_rms, gauss_drift_rms; };
    // rms div B and the drift of the Gauss residual div E - rho from its first
    // value, rho the CIC node charge filtered like J, with the reference's own
    // kernels (its residuals(), simulation_maxwell.hpp:126-166).
    Residuals residuals() {
        const int n = g_.real_size();
        if (rho_.size() == 0) {
            rho_ = DeviceArray<float>(n);
            rres_ = DeviceArray<float>(n);
            r0_ = DeviceArray<float>(n);
        }
        YeeViews v = flds_.views();
        const dim3 tb(16, 16), nb((g_.nx + 15) / 16, (g_.ny + 15) / 16);
        rho_.zero(s_);
        if (parts_.n > 0)
            yee::k_rho_nodes<<<(static_cast<int>(parts_.n) + 255) / 256, 256, 0, s_>>>(parts_.views(), v,
                                                                                      rho_.data(), rp_.qm, 0);
        float* cur = rho_.data();
        float* other = jtmp_.data();
        for (int pass = 0; pass < rp_.jfilter; ++pass) {
            yee::k_binomial3x3<<<nb, tb, 0, s_>>>(cur, other, v);
            std::swap(cur, other);
        }
        if (cur != rho_.data())
            CUDA_CHECK(cudaMemcpyAsync(rho_.data(), cur, static_cast<size_t>(n) * sizeof(float),
                                       cudaMemcpyDeviceToDevice, s_));
        yee::k_gauss_residual<<<nb, tb, 0, s_>>>(v, rho_.data(), rres_.data());
        if (!have_ref_) {
            CUDA_CHECK(cudaMemcpyAsync(r0_.data(), rres_.data(), static_cast<size_t>(n) * sizeof(float),
                                       cudaMemcpyDeviceToDevice, s_));
            have_ref_ = true;
        }
        CUDA_CHECK(cudaMemsetAsync(diag_.data(), 0, diag_.bytes(), s_));
        yee::k_div_stats<<<(n + 255) / 256, 256, 0, s_>>>(v, rres_.data(), r0_.data(), diag_.data());
        CUDA_CHECK(cudaPeekAtLastError());
        double h[2];
        CUDA_CHECK(cudaMemcpyAsync(h, diag_.data(), sizeof(h), cudaMemcpyDeviceToHost, s_));
        s_.synchronize();
        return {std::sqrt(h[0] / n), std::sqrt(h[1] / n)};
    }

    struct WdStats { double sum, rms, max; };
    WdStats wd_stats() { return {0, 0, 0}; }   // no delta-f weights on this path

private:
    Grid       g_;
    RunParams  rp_;
    Particles  parts_;
    YeeFields  flds_;
    CudaStream s_;
    DeviceArray<double> diag_;
    DeviceArray<float>  jtmp_;
    DeviceArray<float>  rho_, rres_, r0_;
    DeviceArray<float>  vcy_, vcz_;
    aw_ctx* ctx_ = nullptr;
    bool inited_ = false;
    bool have_ref_ = false;
    long nstep_ = 0;
};

}  // namespace arc

#endif  // ARC_PIC_SIMULATION_MAXWELL_HPP
