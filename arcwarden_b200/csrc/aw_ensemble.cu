// aw_ensemble.cu — batched ensembles of independent runs (no counterpart in the
// reference, which runs one Simulation at a time).
//
// Each run is an ordinary context on the ensemble's stream with its particle
// SoA owned here. One ensemble step is one CUDA graph. Runs that fill the GPU
// alone are independent child graphs (their whole fused step); the smaller
// runs' grid phases are independent child graphs too, and each of their
// particle phases is ONE launch over the chunks of every small run of that
// model (k_*_multi: block -> (run, chunk) through a device table), so small
// grids fill the machine together. The executor overlaps everything that does
// not depend on each other. Every run computes exactly what it computes alone
// (the same chunk code on the same data).
//
// The autotuner picks, per class of runs (model, grid, particles per cell), the
// spatial re-sort interval and tile size from timed trials on a scratch copy.
#include "aw_internal.h"

#include <algorithm>
#include <map>
#include <memory>
#include <tuple>
#include <vector>

struct aw_ensemble {
    struct Run {
        aw_run_spec spec{};
        aw_ctx* ctx = nullptr;
        void* buf = nullptr;         // x y ux uy uz w (float) + cell (int), each n4 long
        long long n = 0, n4 = 0;
        int tuned_every = -1, tuned_tile = 0;
    };
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::vector<Run> runs;
    cudaGraph_t parent = nullptr;
    cudaGraphExec_t pexec = nullptr;
    std::vector<cudaGraph_t> children;
    std::vector<aw::MultiPhase*> phases;   // the multi-run particle launches of the graph
    long long step = 0;
};

namespace aw {
namespace {

long long run_particles(const aw_run_spec& s) {
    long long ppc = 0;
    for (int k = 0; k < s.nspecies; ++k) ppc += s.species[k].ppc;
    return ppc * static_cast<long long>(s.grid.nx) * s.grid.ny;
}

void drop_ensemble_graph(aw_ensemble& e) {
    if (e.pexec) cudaGraphExecDestroy(e.pexec);
    if (e.parent) cudaGraphDestroy(e.parent);
    for (cudaGraph_t g : e.children) if (g) cudaGraphDestroy(g);
    for (MultiPhase* m : e.phases) multi_free(m);
    e.pexec = nullptr;
    e.parent = nullptr;
    e.children.clear();
    e.phases.clear();
}

// `body` captured on the ensemble's stream into a graph the ensemble owns.
template <class F>
cudaGraph_t capture(aw_ensemble& e, F body) {
    cudaGraph_t g = nullptr;
    AW_CUDA(cudaStreamBeginCapture(e.stream, cudaStreamCaptureModeThreadLocal));
    try {
        body();
    } catch (...) {
        cudaStreamEndCapture(e.stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    AW_CUDA(cudaStreamEndCapture(e.stream, &g));
    e.children.push_back(g);
    return g;
}

// Runs with at least this many chunks fill the GPU's CTA slots on their own
// (148 SMs x 3 CTAs): they keep their whole fused step as one child graph.
constexpr long long kOwnStepChunks = 148LL * 3;

// One ensemble step as one graph. A run large enough to fill the GPU is one
// child graph (its whole fused step), independent of the others. The smaller
// runs share their particle phases: their grid phases are independent child
// graphs, and each particle phase is one multi-run launch over the chunks of
// all small runs of that model, after the grid phases it depends on.
//   ES:     A (solve) -> [push+deposit, small ES runs] -> C (reduction)
//   Darwin: A (E_L, B) -> [dcu deposit, small Darwin runs] -> B (E_T, E)
//           -> [push+deposit, small Darwin runs] -> C
// (Batching every run behind shared phase barriers measured slower: the large
// runs then wait for all grid phases instead of overlapping them.)
void build_ensemble_graph(aw_ensemble& e) {
    AW_CUDA(cudaGraphCreate(&e.parent, 0));
    auto child = [&](cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps) {
        cudaGraphNode_t node;
        AW_CUDA(cudaGraphAddChildGraphNode(&node, e.parent, deps.empty() ? nullptr : deps.data(), deps.size(), g));
        return node;
    };
    std::vector<Ctx*> es, dw;
    std::vector<cudaGraphNode_t> a_es, a_dw;
    for (auto& r : e.runs) {
        Ctx& c = r.ctx->c;
        if ((r.n + kChunk - 1) / kChunk >= kOwnStepChunks) {
            cudaGraph_t g = capture_step_graph(c);
            e.children.push_back(g);
            child(g, {});
            continue;
        }
        const cudaGraphNode_t a = child(capture(e, [&] { step_grid_phase(c, 0); }), {});
        if (c.model == AW_MODEL_ES) { es.push_back(&c); a_es.push_back(a); }
        else { dw.push_back(&c); a_dw.push_back(a); }
    }
    if (!es.empty()) {
        MultiPhase* m = multi_create(kMultiEsPush, es.data(), static_cast<int>(es.size()));
        e.phases.push_back(m);
        const cudaGraphNode_t p = child(capture(e, [&] { multi_launch(m, e.stream); }), a_es);
        for (Ctx* c : es) child(capture(e, [&] { step_grid_phase(*c, 2); }), {p});
    }
    if (!dw.empty()) {
        MultiPhase* md = multi_create(kMultiDcu, dw.data(), static_cast<int>(dw.size()));
        e.phases.push_back(md);
        const cudaGraphNode_t pd = child(capture(e, [&] { multi_launch(md, e.stream); }), a_dw);
        std::vector<cudaGraphNode_t> b;
        for (Ctx* c : dw) b.push_back(child(capture(e, [&] { step_grid_phase(*c, 1); }), {pd}));
        MultiPhase* mm = multi_create(kMultiEmPush, dw.data(), static_cast<int>(dw.size()));
        e.phases.push_back(mm);
        const cudaGraphNode_t pm = child(capture(e, [&] { multi_launch(mm, e.stream); }), b);
        for (Ctx* c : dw) child(capture(e, [&] { step_grid_phase(*c, 2); }), {pm});
    }
    AW_CUDA(cudaGraphInstantiate(&e.pexec, e.parent, 0));
}

float* arr(const aw_ensemble::Run& r, int k) { return static_cast<float*>(r.buf) + static_cast<size_t>(k) * r.n4; }

// Create one run's context and particles on `stream`, loaded by the seeded loader.
void make_run(aw_ensemble::Run& r, const aw_run_spec& s, cudaStream_t stream) {
    r.spec = s;
    need(s.nspecies >= 1 && s.nspecies <= AW_ENSEMBLE_MAX_SPECIES, AW_ERR_ARG, "ensemble: 1..4 species per run");
    r.n = run_particles(s);
    need(r.n > 0, AW_ERR_ARG, "ensemble: a run without particles");
    r.n4 = (r.n + 3) & ~3LL;     // keeps every array 16-byte aligned (bulk-copy chunk loads)
    int rc = aw_ctx_create(&s.grid, &s.params, s.model, stream, &r.ctx);
    if (rc != AW_OK) throw Error(rc, "ensemble: context creation failed");
    // every run takes the two-pass particle kernels: the ensemble's step is
    // faster that way than with the single pass that lone runs above 128
    // particles per cell default to (ensemble64: 22.2 against 31.3 ms)
    const aw_kernel_plan two_pass{0, -1, 0};
    rc = aw_set_kernel_plan(r.ctx, &two_pass);
    if (rc != AW_OK) throw Error(rc, "ensemble: kernel plan");
    AW_CUDA(cudaMalloc(&r.buf, sizeof(float) * 7 * static_cast<size_t>(r.n4)));
    rc = aw_particles_bind(r.ctx, arr(r, 0), arr(r, 1), arr(r, 2), arr(r, 3), arr(r, 4), arr(r, 5),
                           reinterpret_cast<int32_t*>(arr(r, 6)), r.n);
    if (rc != AW_OK) throw Error(rc, "ensemble: particle binding failed");
    rc = aw_load_species(r.ctx, s.species, s.nspecies, s.seed, s.noisy);
    if (rc != AW_OK) throw Error(rc, "ensemble: particle load failed");
}

void free_run(aw_ensemble::Run& r) {
    if (r.ctx) aw_ctx_destroy(r.ctx);
    if (r.buf) cudaFree(r.buf);
    r.ctx = nullptr;
    r.buf = nullptr;
}

void check(int rc) {
    if (rc != AW_OK) {
        char buf[512];
        aw_last_error(buf, sizeof(buf));
        throw Error(rc, buf);
    }
}

// Milliseconds of `fn` on the stream.
template <class F>
float time_on(cudaStream_t s, F fn) {
    cudaEvent_t a, b;
    AW_CUDA(cudaEventCreate(&a));
    AW_CUDA(cudaEventCreate(&b));
    float ms = 0.f;
    try {
        AW_CUDA(cudaEventRecord(a, s));
        fn();
        AW_CUDA(cudaEventRecord(b, s));
        AW_CUDA(cudaEventSynchronize(b));
        AW_CUDA(cudaEventElapsedTime(&ms, a, b));
    } catch (...) {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        throw;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
}

}  // namespace
}  // namespace aw

using aw::Ctx;
using aw::Error;
using aw::guarded;

extern "C" {

int aw_ensemble_create(int32_t nruns, const aw_run_spec* specs, void* stream, aw_ensemble** out) {
    return guarded([&] {
        aw::need(out && (specs || nruns == 0) && nruns >= 0, AW_ERR_ARG, "ensemble_create: bad arguments");
        *out = nullptr;
        std::unique_ptr<aw_ensemble> e(new aw_ensemble());
        if (stream) {
            e->stream = static_cast<cudaStream_t>(stream);
        } else {
            AW_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
            e->own_stream = true;
        }
        e->runs.resize(nruns);
        try {
            for (int r = 0; r < nruns; ++r) aw::make_run(e->runs[r], specs[r], e->stream);
        } catch (...) {
            for (auto& r : e->runs) aw::free_run(r);
            if (e->own_stream) cudaStreamDestroy(e->stream);
            throw;
        }
        *out = e.release();
    });
}

int aw_ensemble_destroy(aw_ensemble* e) {
    if (!e) return AW_OK;
    aw::drop_ensemble_graph(*e);
    for (auto& r : e->runs) aw::free_run(r);
    if (e->own_stream) cudaStreamDestroy(e->stream);
    delete e;
    return AW_OK;
}

int aw_ensemble_init(aw_ensemble* e) {
    return guarded([&] {
        aw::need(e != nullptr, AW_ERR_ARG, "null ensemble");
        aw::drop_ensemble_graph(*e);
        for (auto& r : e->runs) aw::check(aw_init(r.ctx));
        e->step = 0;
    });
}

int aw_ensemble_tune(aw_ensemble* e, int32_t trial_steps) {
    return guarded([&] {
        aw::need(e != nullptr && trial_steps >= 1, AW_ERR_ARG, "ensemble_tune: bad arguments");
        using Key = std::tuple<int, int, int, double, double, long long>;
        std::map<Key, std::pair<int, int>> choice;
        static const int kTiles[3] = {512, 1024, 2048};
        for (auto& run : e->runs) {
            const aw_run_spec& s = run.spec;
            const Key key{s.model, s.grid.nx, s.grid.ny, s.grid.Lx, s.grid.Ly, run.n};
            auto it = choice.find(key);
            if (it == choice.end()) {
                // a scratch copy of the run: warm it up so the particles have mixed, then time the
                // candidates from the same state (each re-sort permutes; the physics is order-free)
                aw_ensemble::Run t;
                try {
                    aw::make_run(t, s, e->stream);
                    aw::check(aw_init(t.ctx));
                    Ctx& c = t.ctx->c;
                    aw::check(aw_set_resort(t.ctx, 0));
                    aw::check(aw_run(t.ctx, 0, trial_steps, 1));
                    long long n0 = trial_steps;
                    auto steps_ms = [&] {
                        const float ms = aw::time_on(e->stream, [&] { aw::check(aw_run(t.ctx, n0, trial_steps, 1)); });
                        n0 += trial_steps;
                        return ms / trial_steps;
                    };
                    float best = steps_ms();
                    int best_every = 0, best_tile = aw::kChunk / 2;
                    for (int tile : kTiles) {
                        c.resort_tile = tile;
                        const float rs = aw::time_on(e->stream, [&] { aw::check(aw_resort(t.ctx)); });
                        const float st = steps_ms();
                        // amortised over a 50-step interval, the re-sort must buy back its cost
                        const float cost = st + rs / 50.0f;
                        if (cost < best) { best = cost; best_every = 50; best_tile = tile; }
                    }
                    it = choice.emplace(key, std::make_pair(best_every, best_tile)).first;
                } catch (...) {
                    aw::free_run(t);
                    throw;
                }
                aw::free_run(t);
            }
            run.tuned_every = it->second.first;
            run.tuned_tile = it->second.second;
            run.ctx->c.resort_every = run.tuned_every;
            run.ctx->c.resort_tile = run.tuned_tile;
        }
        aw::drop_ensemble_graph(*e);
    });
}

int aw_ensemble_tuning(aw_ensemble* e, int32_t run, int32_t* resort_every, int32_t* resort_tile) {
    return guarded([&] {
        aw::need(e && resort_every && resort_tile, AW_ERR_ARG, "null argument");
        aw::need(run >= 0 && run < static_cast<int32_t>(e->runs.size()), AW_ERR_ARG, "ensemble: run out of range");
        *resort_every = e->runs[run].ctx->c.resort_every;
        *resort_tile = e->runs[run].ctx->c.resort_tile;
    });
}

int aw_ensemble_run(aw_ensemble* e, int64_t nsteps, int32_t concurrent) {
    return guarded([&] {
        aw::need(e != nullptr && nsteps >= 0, AW_ERR_ARG, "ensemble_run: bad arguments");
        if (!concurrent) {
            for (auto& r : e->runs) aw::check(aw_run(r.ctx, e->step, nsteps, 1));
            e->step += nsteps;
            return;
        }
        for (auto& r : e->runs) {
            aw::prepare_step(r.ctx->c);
            aw::launch_set_step(r.ctx->c, e->step);
        }
        if (!e->pexec) {
            try {
                aw::build_ensemble_graph(*e);
            } catch (...) {
                aw::drop_ensemble_graph(*e);
                throw;
            }
        }
        for (int64_t i = 0; i < nsteps; ++i) {
            const int64_t s = e->step + i;
            for (auto& r : e->runs) {
                Ctx& c = r.ctx->c;
                if (c.resort_every > 0 && s > 0 && s % c.resort_every == 0) aw::launch_resort(c);
            }
            AW_CUDA(cudaGraphLaunch(e->pexec, e->stream));
        }
        e->step += nsteps;
    });
}

int aw_ensemble_diag(aw_ensemble* e, int32_t run, aw_diag* out) {
    return guarded([&] {
        aw::need(e && out, AW_ERR_ARG, "null argument");
        aw::need(run >= 0 && run < static_cast<int32_t>(e->runs.size()), AW_ERR_ARG, "ensemble: run out of range");
        aw::check(aw_step_diag(e->runs[run].ctx, out));
    });
}

int aw_ensemble_particles(aw_ensemble* e, int32_t run, float** x, float** y, float** ux, float** uy, float** uz,
                          float** w, int64_t* n) {
    return guarded([&] {
        aw::need(e && x && y && ux && uy && uz && w && n, AW_ERR_ARG, "null argument");
        aw::need(run >= 0 && run < static_cast<int32_t>(e->runs.size()), AW_ERR_ARG, "ensemble: run out of range");
        const auto& r = e->runs[run];
        *x = aw::arr(r, 0); *y = aw::arr(r, 1); *ux = aw::arr(r, 2); *uy = aw::arr(r, 3); *uz = aw::arr(r, 4);
        *w = aw::arr(r, 5);
        *n = r.n;
    });
}

}  // extern "C"
