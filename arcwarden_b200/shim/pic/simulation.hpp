// pic/simulation.hpp (B200 shim) — Simulation<Cfg> (include/pic/simulation.hpp:
// 41-126) on libarcb200's fused step. init() loads the particles, allocates the
// reference's Sources/Fields, creates a library context bound to them and runs
// aw_init; every step() is one replay of the captured step graph (aw_run),
// and a dump step enqueues an asynchronous copy of the step's GPU-reduced
// diagnostics (the shim's pic/diagnostics.hpp), with no host sync.
// With ARCB200_LOOP_TIME set in the environment, the destructor prints to
// stderr the wall time from the first step() to its own start, after a stream
// sync: the step loop and whatever the caller did between and after the steps
// (a runner's diagnostics and their files), without the start-up.
#ifndef ARC_PIC_SIMULATION_HPP
#define ARC_PIC_SIMULATION_HPP

#include "pic/config.hpp"
#include "pic/cuda_utils.hpp"
#include "pic/depositor.hpp"
#include "pic/diagnostics.hpp"
#include "pic/fields.hpp"
#include "pic/grid.hpp"
#include "pic/particles.hpp"
#include "pic/pump.hpp"
#include "pic/pusher.hpp"
#include "pic/solver_darwin.hpp"
#include "pic/solver_es.hpp"
#include "pic/sources.hpp"
#include "pic/species.hpp"
#include "pic/spectral.hpp"

#include "../arcb200_shim.hpp"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>

namespace arc {

template <class Cfg = arc::Cfg>
class Simulation {
public:
    Simulation(const Grid& g, const RunParams& rp, const std::string& csv = "")
        : p_(rp), grid_(g), spectral_(g), diag_(csv) {
        diag_.set_geometry(g.dx, g.dy);
    }
    Simulation(const Grid& g, const RunParams& rp, const SpeciesList& species, const std::string& csv = "")
        : p_(rp), grid_(g), species_(species), spectral_(g), diag_(csv) {
        diag_.set_geometry(g.dx, g.dy);
    }
    ~Simulation() {
        if (steps_ > 0 && std::getenv("ARCB200_LOOP_TIME")) try {
            stream_.synchronize();
            const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - first_step_).count();
            std::fprintf(stderr, "arcb200 loop: %ld steps in %.6f s\n", steps_, s);
        } catch (...) {}
        if (ctx_) aw_ctx_destroy(ctx_);
    }
    Simulation(const Simulation&) = delete;
    Simulation& operator=(const Simulation&) = delete;

    static constexpr bool darwin() { return Cfg::field_model == FieldModel::Darwin; }

    // Load, allocate, t = 0 fields (and, for ES, the half-step velocity rollback).
    void init() {
        if (!species_.empty()) particles_.initialize(species_, grid_, p_, stream_);
        else particles_.initialize(p_, grid_, stream_);
        sources_.allocate(grid_);
        fields_.allocate(grid_);
        if constexpr (darwin()) {
            sources_.allocate_em(grid_);
            fields_.allocate_em(grid_, stream_);
            spectral_.enable_em();
        }
        if (!ctx_) {
            const aw_grid ag = shim::grid_of(grid_);
            const aw_params ap = shim::params(p_, Cfg::has_b0);
            shim::check(aw_ctx_create(&ag, &ap, darwin() ? AW_MODEL_DARWIN : AW_MODEL_ES, stream_.get(), &ctx_),
                        "ctx_create");
        }
        particles_.bind(ctx_);
        shim::bind_sources(ctx_, sources_);
        shim::bind_fields(ctx_, fields_);
        shim::check(aw_init(ctx_), "init");
        shim::check(aw_step_diag_device(ctx_, &dev_diag_), "step_diag_device");
    }

    // One PIC step (the fused graph), then the diagnostics when due
    // (Diagnostics::maybe_compute's cadence: dump_every <= 0 means every step).
    void step(long n) {
        if (steps_++ == 0) first_step_ = std::chrono::steady_clock::now();
        shim::check(aw_run(ctx_, n, 1, 1), "run");
        if (p_.dump_every <= 0 || n % p_.dump_every == 0) diag_.record_async(n, n * p_.dt, dev_diag_, stream_);
    }

    void run() {
        for (long n = 0; n < p_.nsteps; ++n) step(n);
        stream_.synchronize();
        diag_.drain();
    }

    // The Darwin field solve for the current particle state, from the separate
    // operators (deposits, E_L + B, dcu, E_T, E_total + pump).
    void darwin_fields(double t, cudaStream_t s) {
        sources_.zero_rho_j(s);
        sources_.zero_dcu_amu(s);
        Depositor<Cfg>::charge_current_sorted(particles_, sources_, grid_, p_, s);
        Depositor<Cfg>::deposit_amu(particles_, sources_, grid_, p_, s);
        dsolver_.solve_el_b(sources_, fields_, spectral_, p_, s);
        add_background_b0(fields_, grid_, p_, s);
        dsolver_.form_el(fields_, s);
        add_pump_field(fields_, grid_, p_, t, s);
        sources_.zero_dcu(s);
        Depositor<Cfg>::deposit_dcu(particles_, sources_, fields_, grid_, p_, s);
        dsolver_.solve_et(sources_, fields_, spectral_, p_, s);
        dsolver_.form_etotal(fields_, s);
        add_pump_field(fields_, grid_, p_, t, s);
    }

    const Diagnostics& diagnostics() const { return diag_; }
    const Fields&      fields() const { return fields_; }
    const RunParams&   params() const { return p_; }
    const Particles&   particles() const { return particles_; }
    Particles&         particles() { return particles_; }
    const Grid&        grid() const { return grid_; }

private:
    RunParams      p_;
    Grid           grid_;
    SpeciesList    species_;
    Particles      particles_;
    Sources        sources_;
    Fields         fields_;
    SpectralEngine spectral_;
    ElectrostaticSpectralSolver solver_;
    DarwinSpectralSolver        dsolver_;
    Diagnostics    diag_;
    CudaStream     stream_;
    aw_ctx*        ctx_ = nullptr;
    const aw_diag* dev_diag_ = nullptr;
    long           steps_ = 0;
    std::chrono::steady_clock::time_point first_step_{};
};

}  // namespace arc

#endif  // ARC_PIC_SIMULATION_HPP
