// ref_harness.cu — C entry points over the reference's OWN CUDA implementation.
//
// TEST INFRASTRUCTURE ONLY. Built by `make -C oracle ref` into oracle/_ref/
// (git-ignored) from the ArcWarden headers where they lie (-I <reference>/include);
// no reference source is copied into this repository. Used by the GPU parity
// tests (the reference's CUDA path on identical seeded particles) and by
// `bench.py --impl reference` (the reference's Simulation step timed on the GPU).
//
// Everything here calls the reference's public C++ API unchanged:
// Simulation<Cfg>/Simulation<CfgDarwin> (include/pic/simulation.hpp),
// MaxwellSimulation (include/pic/simulation_maxwell.hpp: the Yee branch),
// Particles::initialize / sort_by_tile / build_tile_bins (particles.hpp),
// Depositor<Cfg> (depositor.hpp), Pusher<Cfg> (pusher.hpp), the spectral solvers
// (solver_es.hpp, solver_darwin.hpp) and add_background_b0/add_pump_field (pump.hpp).
#include "pic/config.hpp"
#include "pic/cuda_utils.hpp"
#include "pic/depositor.hpp"
#include "pic/fields.hpp"
#include "pic/grid.hpp"
#include "pic/particles.hpp"
#include "pic/pump.hpp"
#include "pic/pusher.hpp"
#include "pic/simulation.hpp"
#include "pic/simulation_maxwell.hpp"
#include "pic/solver_darwin.hpp"
#include "pic/solver_es.hpp"
#include "pic/sources.hpp"
#include "pic/spectral.hpp"
#include "pic/species.hpp"

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace arc;
using CfgGlobal = SimConfig<2, 3, ShapeOrder::CIC, float, true, AtomicGlobalDeposit>;
using CfgTiled = SimConfig<2, 3, ShapeOrder::CIC, float, true, TiledBinnedDeposit>;

struct ref_params {
    double dt, qm, eps0, n0, c;
    float B0[3];
    int pump;
    double pump_ex, pump_ey, pump_ez, pump_k0, pump_w0, pump_trmp, pump_toff;
};
struct ref_species {
    int ppc;
    double density;
    double uth[3], ufl[3];
};

static thread_local std::string g_err;
extern "C" const char* ref_last_error() { return g_err.c_str(); }

template <class F>
static int guard(F&& f) {
    try { f(); return 0; }
    catch (const std::exception& e) { g_err = e.what(); return -1; }
}

static RunParams make_rp(const ref_params* p, int noisy, unsigned long seed) {
    RunParams rp;
    rp.dt = p->dt; rp.qm = p->qm; rp.eps0 = p->eps0; rp.n0 = p->n0; rp.c = p->c;
    for (int d = 0; d < 3; ++d) rp.B0[d] = p->B0[d];
    rp.pump = p->pump != 0;
    rp.pump_ex = p->pump_ex; rp.pump_ey = p->pump_ey; rp.pump_ez = p->pump_ez;
    rp.pump_k0 = p->pump_k0; rp.pump_w0 = p->pump_w0;
    rp.pump_trmp = p->pump_trmp; rp.pump_toff = p->pump_toff;
    rp.noisy_load = noisy != 0;
    rp.rng_seed = seed;
    rp.dump_every = 1L << 30;     // keep host diagnostics out of the step
    return rp;
}
static SpeciesList make_sp(const ref_species* sp, int nsp) {
    SpeciesList l;
    for (int i = 0; i < nsp; ++i) {
        Species s;
        s.name = "s" + std::to_string(i);
        s.density = sp[i].density;
        s.ppc = sp[i].ppc;
        for (int d = 0; d < 3; ++d) { s.uth[d] = sp[i].uth[d]; s.ufl[d] = sp[i].ufl[d]; }
        l.push_back(s);
    }
    return l;
}

// ---- whole-simulation handle ------------------------------------------------
struct RefSim {
    int model;
    Grid g;
    RunParams rp;
    Simulation<Cfg>* es = nullptr;
    Simulation<CfgDarwin>* dw = nullptr;
    ~RefSim() { delete es; delete dw; }
    Particles& parts() { return es ? es->particles() : dw->particles(); }
    const Fields& fields() const { return es ? es->fields() : dw->fields(); }
};

extern "C" void* ref_create(int model, int nx, int ny, double Lx, double Ly, const ref_params* p,
                 const ref_species* sp, int nsp, int noisy, unsigned long seed) {
    RefSim* h = nullptr;
    int rc = guard([&] {
        h = new RefSim();
        h->model = model;
        h->g = Grid(nx, ny, Lx, Ly);
        h->rp = make_rp(p, noisy, seed);
        SpeciesList l = make_sp(sp, nsp);
        if (model == 0) h->es = new Simulation<Cfg>(h->g, h->rp, l);
        else h->dw = new Simulation<CfgDarwin>(h->g, h->rp, l);
    });
    if (rc) { delete h; return nullptr; }
    return h;
}
extern "C" void ref_destroy(void* hv) { delete static_cast<RefSim*>(hv); }

extern "C" int ref_init(void* hv) {
    return guard([&] {
        RefSim* h = static_cast<RefSim*>(hv);
        if (h->es) h->es->init(); else h->dw->init();
    });
}
extern "C" int ref_step(void* hv, long n) {
    return guard([&] {
        RefSim* h = static_cast<RefSim*>(hv);
        if (h->es) h->es->step(n); else h->dw->step(n);
        CUDA_CHECK(cudaDeviceSynchronize());
    });
}
// Times `nsteps` steps starting at n0 with CUDA events on the default stream
// bracketing a device sync (the Simulation owns its own stream).
extern "C" int ref_time_steps(void* hv, long n0, long nsteps, float* ms) {
    return guard([&] {
        RefSim* h = static_cast<RefSim*>(hv);
        CUDA_CHECK(cudaDeviceSynchronize());
        CudaEvent a, b;
        a.record(nullptr);
        for (long i = 0; i < nsteps; ++i) {
            if (h->es) h->es->step(n0 + i); else h->dw->step(n0 + i);
        }
        CUDA_CHECK(cudaDeviceSynchronize());
        b.record(nullptr);
        b.synchronize();
        *ms = b.elapsed_ms_since(a);
    });
}
extern "C" long ref_n(void* hv) { return static_cast<long>(static_cast<RefSim*>(hv)->parts().n); }

static int copy_down(const void* dptr, void* host, size_t bytes) {
    if (!dptr) return -2;
    CUDA_CHECK(cudaDeviceSynchronize());
    CUDA_CHECK(cudaMemcpy(host, dptr, bytes, cudaMemcpyDeviceToHost));
    return 0;
}

// Copy a particle array or a field (as the reference holds it) to host memory.
extern "C" int ref_get(void* hv, const char* name, void* host) {
    int out = 0;
    int rc = guard([&] {
        RefSim* h = static_cast<RefSim*>(hv);
        Particles& P = h->parts();
        const Fields& F = h->fields();
        const size_t n = P.n, nc = static_cast<size_t>(h->g.real_size());
        const std::string s(name);
        if (s == "x") out = copy_down(P.x.data(), host, n * 4);
        else if (s == "y") out = copy_down(P.y.data(), host, n * 4);
        else if (s == "ux") out = copy_down(P.ux.data(), host, n * 4);
        else if (s == "uy") out = copy_down(P.uy.data(), host, n * 4);
        else if (s == "uz") out = copy_down(P.uz.data(), host, n * 4);
        else if (s == "w") out = copy_down(P.w.data(), host, n * 4);
        else if (s == "cell") out = copy_down(P.cell.data(), host, n * 4);
        else if (s == "Ex") out = copy_down(F.Ex.data(), host, nc * 4);
        else if (s == "Ey") out = copy_down(F.Ey.data(), host, nc * 4);
        else if (s == "Ez") out = copy_down(F.Ez.data(), host, nc * 4);
        else if (s == "Bx") out = copy_down(F.Bx.data(), host, nc * 4);
        else if (s == "By") out = copy_down(F.By.data(), host, nc * 4);
        else if (s == "Bz") out = copy_down(F.Bz.data(), host, nc * 4);
        else if (s == "ELx") out = copy_down(F.ELx.data(), host, nc * 4);
        else if (s == "ELy") out = copy_down(F.ELy.data(), host, nc * 4);
        else if (s == "ETx") out = copy_down(F.ETx.data(), host, nc * 4);
        else if (s == "ETy") out = copy_down(F.ETy.data(), host, nc * 4);
        else if (s == "ETz") out = copy_down(F.ETz.data(), host, nc * 4);
        else out = -3;
    });
    return rc ? rc : out;
}

// Overwrite the reference simulation's particles from host arrays (cell is
// recomputed by Particles::migrate).
extern "C" int ref_set_particles(void* hv, const float* x, const float* y, const float* ux, const float* uy,
                      const float* uz, const float* w) {
    return guard([&] {
        RefSim* h = static_cast<RefSim*>(hv);
        Particles& P = h->parts();
        const size_t b = P.n * sizeof(float);
        CUDA_CHECK(cudaMemcpy(P.x.data(), x, b, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMemcpy(P.y.data(), y, b, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMemcpy(P.ux.data(), ux, b, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMemcpy(P.uy.data(), uy, b, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMemcpy(P.uz.data(), uz, b, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMemcpy(P.w.data(), w, b, cudaMemcpyHostToDevice));
        CudaStream s;
        P.migrate(h->g, s);
        s.synchronize();
    });
}

// ---- operator-level calls on standalone containers ----------------------------
// Load particles with the reference loader (Particles::initialize(SpeciesList...)).
extern "C" int ref_load(int nx, int ny, double Lx, double Ly, const ref_species* sp, int nsp, int noisy,
             unsigned long seed, float* x, float* y, float* ux, float* uy, float* uz, float* w, int* cell) {
    return guard([&] {
        Grid g(nx, ny, Lx, Ly);
        ref_params p{};
        p.dt = 0.1; p.qm = -1; p.eps0 = 1; p.n0 = 1; p.c = 1;
        RunParams rp = make_rp(&p, noisy, seed);
        CudaStream s;
        Particles P;
        P.initialize(make_sp(sp, nsp), g, rp, s);
        s.synchronize();
        const size_t b = P.n * 4;
        CUDA_CHECK(cudaMemcpy(x, P.x.data(), b, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(y, P.y.data(), b, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(ux, P.ux.data(), b, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(uy, P.uy.data(), b, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(uz, P.uz.data(), b, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(w, P.w.data(), b, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(cell, P.cell.data(), b, cudaMemcpyDeviceToHost));
    });
}

// The single-species RunParams load, Particles::initialize(rp, g, s).
// f[] = weight, vth, vd, beam_frac, beam_vd, beam_vth, perturb_amp;
// i[] = ppc, two_stream, bump_on_tail, perturb_kx, noisy.
extern "C" int ref_load_legacy(int nx, int ny, double Lx, double Ly, const double* f, const int* i,
             unsigned long seed, float* x, float* y, float* ux, float* uy, float* uz, float* w, int* cell) {
    return guard([&] {
        Grid g(nx, ny, Lx, Ly);
        ref_params p{};
        p.dt = 0.1; p.qm = -1; p.eps0 = 1; p.n0 = 1; p.c = 1;
        RunParams rp = make_rp(&p, i[4], seed);
        rp.weight = f[0]; rp.vth = f[1]; rp.vd = f[2];
        rp.beam_frac = f[3]; rp.beam_vd = f[4]; rp.beam_vth = f[5]; rp.perturb_amp = f[6];
        rp.ppc = i[0]; rp.two_stream = i[1] != 0; rp.bump_on_tail = i[2] != 0; rp.perturb_kx = i[3];
        CudaStream s;
        Particles P;
        P.initialize(rp, g, s);
        s.synchronize();
        const size_t b = P.n * 4;
        CUDA_CHECK(cudaMemcpy(x, P.x.data(), b, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(y, P.y.data(), b, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(ux, P.ux.data(), b, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(uy, P.uy.data(), b, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(uz, P.uz.data(), b, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(w, P.w.data(), b, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(cell, P.cell.data(), b, cudaMemcpyDeviceToHost));
    });
}

static void upload(Particles& P, long n, const float* x, const float* y, const float* ux,
                   const float* uy, const float* uz, const float* w, const Grid& g, cudaStream_t s) {
    P.allocate_n(static_cast<size_t>(n));
    const size_t b = n * sizeof(float);
    CUDA_CHECK(cudaMemcpy(P.x.data(), x, b, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(P.y.data(), y, b, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(P.ux.data(), ux, b, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(P.uy.data(), uy, b, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(P.uz.data(), uz, b, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(P.w.data(), w, b, cudaMemcpyHostToDevice));
    P.migrate(g, s);
}

// Deposit with the reference policies: which = 0 global-atomic rho, 1 Cfg (ES
// default dispatch) rho, 2 tiled rho, 3 Darwin rho+J (charge_current),
// 4 Darwin sorted rho+J, 5 amu (after a sort), 6 dcu (after a sort; fields from
// `f6` = Ex,Ey,Ez,Bx,By,Bz host arrays). out: rho[,Jx,Jy,Jz] or amu0..3 or dcu.
extern "C" int ref_deposit(int which, int nx, int ny, double Lx, double Ly, double qm, long n, const float* x,
                const float* y, const float* ux, const float* uy, const float* uz, const float* w,
                const float* f6, float* out) {
    return guard([&] {
        Grid g(nx, ny, Lx, Ly);
        ref_params p{};
        p.dt = 0.1; p.qm = qm; p.eps0 = 1; p.n0 = 1; p.c = 1;
        RunParams rp = make_rp(&p, 1, 0);
        CudaStream s;
        Particles P;
        upload(P, n, x, y, ux, uy, uz, w, g, s);
        Sources src(g);
        src.allocate_em(g);
        src.zero_rho_j(s);
        src.zero_dcu_amu(s);
        const size_t nc = g.real_size(), b = nc * 4;
        auto down = [&](const DeviceArray<float>& a, float* o) {
            s.synchronize();
            CUDA_CHECK(cudaMemcpy(o, a.data(), b, cudaMemcpyDeviceToHost));
        };
        if (which == 0) { Depositor<CfgGlobal>::charge(P, src, g, rp, s); down(src.rho, out); }
        else if (which == 1) { Depositor<Cfg>::charge(P, src, g, rp, s); down(src.rho, out); }
        else if (which == 2) { Depositor<CfgTiled>::charge(P, src, g, rp, s); down(src.rho, out); }
        else if (which == 3 || which == 4) {
            if (which == 3) Depositor<CfgDarwin>::charge_current(P, src, g, rp, s);
            else Depositor<CfgDarwin>::charge_current_sorted(P, src, g, rp, s);
            down(src.rho, out); down(src.Jx, out + nc); down(src.Jy, out + 2 * nc); down(src.Jz, out + 3 * nc);
        } else if (which == 5) {
            P.sort_by_tile(g, 16, 16, s);
            Depositor<CfgDarwin>::deposit_amu(P, src, g, rp, s);
            down(src.amu0, out); down(src.amu1, out + nc); down(src.amu2, out + 2 * nc); down(src.amu3, out + 3 * nc);
        } else if (which == 6) {
            Fields F(g);
            F.allocate_em(g, s);
            DeviceArray<float>* fa[6] = {&F.Ex, &F.Ey, &F.Ez, &F.Bx, &F.By, &F.Bz};
            for (int k = 0; k < 6; ++k) CUDA_CHECK(cudaMemcpy(fa[k]->data(), f6 + k * nc, b, cudaMemcpyHostToDevice));
            P.sort_by_tile(g, 16, 16, s);
            Depositor<CfgDarwin>::deposit_dcu(P, src, F, g, rp, s);
            down(src.dcux, out); down(src.dcuy, out + nc); down(src.dcuz, out + 2 * nc);
        } else {
            throw std::runtime_error("ref_deposit: bad policy");
        }
    });
}

// Push with the reference pushers on given fields. which = 0 ES boris (then
// migrate = 0/1), 1 EM push (after a tile sort; particle order is permuted),
// 2 half_step_back. f6 = Ex,Ey[,Ez,Bx,By,Bz]; particle arrays are in/out.
extern "C" int ref_push(int which, int nx, int ny, double Lx, double Ly, const ref_params* p, long n, float* x,
             float* y, float* ux, float* uy, float* uz, float* w, const float* f6, int do_migrate) {
    return guard([&] {
        Grid g(nx, ny, Lx, Ly);
        RunParams rp = make_rp(p, 1, 0);
        CudaStream s;
        Particles P;
        upload(P, n, x, y, ux, uy, uz, w, g, s);
        Fields F(g);
        F.allocate_em(g, s);
        const size_t nc = g.real_size(), b = nc * 4;
        DeviceArray<float>* fa[6] = {&F.Ex, &F.Ey, &F.Ez, &F.Bx, &F.By, &F.Bz};
        const int nf = (which == 1) ? 6 : 2;
        for (int k = 0; k < nf; ++k) CUDA_CHECK(cudaMemcpy(fa[k]->data(), f6 + k * nc, b, cudaMemcpyHostToDevice));
        if (which == 0) Pusher<Cfg>::boris(P, F, g, rp, s);
        else if (which == 2) Pusher<Cfg>::half_step_back(P, F, g, rp, s);
        else {
            P.sort_by_tile(g, 16, 16, s);
            Pusher<CfgDarwin>::boris_em(P, F, g, rp, s);
        }
        if (do_migrate) P.migrate(g, s);
        s.synchronize();
        const size_t bb = P.n * 4;
        CUDA_CHECK(cudaMemcpy(x, P.x.data(), bb, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(y, P.y.data(), bb, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(ux, P.ux.data(), bb, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(uy, P.uy.data(), bb, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(uz, P.uz.data(), bb, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(w, P.w.data(), bb, cudaMemcpyDeviceToHost));
    });
}

// Spectral solves. which = 0 ES (rho -> Ex,Ey); 1 Darwin solve_el_b
// (rho,Jx,Jy,Jz -> ELx,ELy,Bx,By,Bz); 2 solve_et (dcu x3, amu x4 -> ETx,ETy,ETz).
extern "C" int ref_solve(int which, int nx, int ny, double Lx, double Ly, const ref_params* p, const float* in,
              float* out) {
    return guard([&] {
        Grid g(nx, ny, Lx, Ly);
        RunParams rp = make_rp(p, 1, 0);
        CudaStream s;
        Sources src(g);
        src.allocate_em(g);
        Fields F(g);
        F.allocate_em(g, s);
        SpectralEngine eng(g);
        eng.enable_em();
        const size_t nc = g.real_size(), b = nc * 4;
        auto up = [&](DeviceArray<float>& a, const float* h) { CUDA_CHECK(cudaMemcpy(a.data(), h, b, cudaMemcpyHostToDevice)); };
        auto down = [&](const DeviceArray<float>& a, float* o) { s.synchronize(); CUDA_CHECK(cudaMemcpy(o, a.data(), b, cudaMemcpyDeviceToHost)); };
        if (which == 0) {
            up(src.rho, in);
            ElectrostaticSpectralSolver().solve(src, F, eng, rp, s);
            down(F.Ex, out); down(F.Ey, out + nc);
        } else if (which == 1) {
            up(src.rho, in); up(src.Jx, in + nc); up(src.Jy, in + 2 * nc); up(src.Jz, in + 3 * nc);
            DarwinSpectralSolver().solve_el_b(src, F, eng, rp, s);
            down(F.ELx, out); down(F.ELy, out + nc); down(F.Bx, out + 2 * nc); down(F.By, out + 3 * nc); down(F.Bz, out + 4 * nc);
        } else if (which == 2) {
            up(src.dcux, in); up(src.dcuy, in + nc); up(src.dcuz, in + 2 * nc);
            up(src.amu0, in + 3 * nc); up(src.amu1, in + 4 * nc); up(src.amu2, in + 5 * nc); up(src.amu3, in + 6 * nc);
            DarwinSpectralSolver().solve_et(src, F, eng, rp, s);
            down(F.ETx, out); down(F.ETy, out + nc); down(F.ETz, out + 2 * nc);
        } else {
            throw std::runtime_error("ref_solve: bad solver");
        }
    });
}

// Tile binning (Particles::build_tile_bins / sort_by_tile): off[ntiles+1] and,
// for the index binning, idx[n]; for the physical sort the permuted x array.
extern "C" int ref_bins(int physical, int nx, int ny, double Lx, double Ly, long n, const float* x, const float* y,
             int tx, int ty, int* off, int* idx_or_cell) {
    return guard([&] {
        Grid g(nx, ny, Lx, Ly);
        CudaStream s;
        Particles P;
        std::vector<float> zero(n, 0.0f), one(n, 1.0f);
        upload(P, n, x, y, zero.data(), zero.data(), zero.data(), one.data(), g, s);
        if (physical) P.sort_by_tile(g, tx, ty, s); else P.build_tile_bins(g, tx, ty, s);
        s.synchronize();
        CUDA_CHECK(cudaMemcpy(off, P.bin_off.data(), (P.bin_ntiles + 1) * 4, cudaMemcpyDeviceToHost));
        if (physical) CUDA_CHECK(cudaMemcpy(idx_or_cell, P.cell.data(), n * 4, cudaMemcpyDeviceToHost));
        else CUDA_CHECK(cudaMemcpy(idx_or_cell, P.bin_idx.data(), n * 4, cudaMemcpyDeviceToHost));
    });
}


// ---- the Yee branch (MaxwellSimulation, include/pic/simulation_maxwell.hpp) ----
// Particles from host arrays (cell recomputed by Particles::migrate); fields
// start at zero as the reference's YeeFields do. tile_sort = 0: the flat
// push + Esirkepov + migrate path; > 0: the tiled path with a physical sort
// every tile_sort steps.
struct RefYee {
    Grid g;
    RunParams rp;
    MaxwellSimulation* sim = nullptr;
    ~RefYee() { delete sim; }
};

extern "C" void* ref_yee_create(int nx, int ny, double Lx, double Ly, const ref_params* p, int tile_sort,
                                int jfilter, long n, const float* x, const float* y, const float* ux, const float* uy,
                                const float* uz, const float* w) {
    RefYee* h = nullptr;
    int rc = guard([&] {
        h = new RefYee();
        h->g = Grid(nx, ny, Lx, Ly);
        h->rp = make_rp(p, 0, 0);
        h->rp.tile_sort = tile_sort;
        h->rp.jfilter = jfilter;
        h->sim = new MaxwellSimulation(h->g, h->rp);
        Particles& P = h->sim->particles();
        P.allocate_n(static_cast<std::size_t>(n));
        const size_t b = static_cast<size_t>(n) * sizeof(float);
        CUDA_CHECK(cudaMemcpy(P.x.data(), x, b, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMemcpy(P.y.data(), y, b, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMemcpy(P.ux.data(), ux, b, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMemcpy(P.uy.data(), uy, b, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMemcpy(P.uz.data(), uz, b, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMemcpy(P.w.data(), w, b, cudaMemcpyHostToDevice));
        P.migrate(h->g, h->sim->stream());
        h->sim->stream().synchronize();
    });
    if (rc) { delete h; return nullptr; }
    return h;
}
// The same, with the particles from the reference's own seeded loader
// (Particles::initialize(SpeciesList, Grid, RunParams, stream)).
extern "C" void* ref_yee_create_species(int nx, int ny, double Lx, double Ly, const ref_params* p, int tile_sort,
                                        int jfilter, const ref_species* sp, int nsp, int noisy, unsigned long seed) {
    RefYee* h = nullptr;
    int rc = guard([&] {
        h = new RefYee();
        h->g = Grid(nx, ny, Lx, Ly);
        h->rp = make_rp(p, noisy, seed);
        h->rp.tile_sort = tile_sort;
        h->rp.jfilter = jfilter;
        h->sim = new MaxwellSimulation(h->g, h->rp);
        h->sim->particles().initialize(make_sp(sp, nsp), h->g, h->rp, h->sim->stream());
        h->sim->stream().synchronize();
    });
    if (rc) { delete h; return nullptr; }
    return h;
}
extern "C" long ref_yee_n(void* hv) { return static_cast<long>(static_cast<RefYee*>(hv)->sim->particles().n); }
extern "C" void ref_yee_destroy(void* hv) { delete static_cast<RefYee*>(hv); }

extern "C" int ref_yee_step(void* hv, long nsteps) {
    return guard([&] {
        RefYee* h = static_cast<RefYee*>(hv);
        for (long i = 0; i < nsteps; ++i) h->sim->step();
        h->sim->stream().synchronize();
    });
}

extern "C" int ref_yee_time_steps(void* hv, long nsteps, float* ms) {
    return guard([&] {
        RefYee* h = static_cast<RefYee*>(hv);
        h->sim->stream().synchronize();
        CudaEvent a, b;
        a.record(h->sim->stream());
        for (long i = 0; i < nsteps; ++i) h->sim->step();
        b.record(h->sim->stream());
        b.synchronize();
        *ms = b.elapsed_ms_since(a);
    });
}

extern "C" int ref_yee_get(void* hv, const char* name, void* host) {
    int out = 0;
    int rc = guard([&] {
        RefYee* h = static_cast<RefYee*>(hv);
        h->sim->stream().synchronize();
        Particles& P = h->sim->particles();
        YeeFields& F = h->sim->fields();
        const size_t n = P.n, nc = static_cast<size_t>(h->g.real_size());
        const std::string s(name);
        if (s == "x") out = copy_down(P.x.data(), host, n * 4);
        else if (s == "y") out = copy_down(P.y.data(), host, n * 4);
        else if (s == "ux") out = copy_down(P.ux.data(), host, n * 4);
        else if (s == "uy") out = copy_down(P.uy.data(), host, n * 4);
        else if (s == "uz") out = copy_down(P.uz.data(), host, n * 4);
        else if (s == "w") out = copy_down(P.w.data(), host, n * 4);
        else if (s == "Ex") out = copy_down(F.ex_.data(), host, nc * 4);
        else if (s == "Ey") out = copy_down(F.ey_.data(), host, nc * 4);
        else if (s == "Ez") out = copy_down(F.ez_.data(), host, nc * 4);
        else if (s == "Bx") out = copy_down(F.bx_.data(), host, nc * 4);
        else if (s == "By") out = copy_down(F.by_.data(), host, nc * 4);
        else if (s == "Bz") out = copy_down(F.bz_.data(), host, nc * 4);
        else if (s == "Jx") out = copy_down(F.jx_.data(), host, nc * 4);
        else if (s == "Jy") out = copy_down(F.jy_.data(), host, nc * 4);
        else if (s == "Jz") out = copy_down(F.jz_.data(), host, nc * 4);
        else out = -3;
    });
    return rc ? rc : out;
}
