// pic/diag/manager.hpp (B200 shim) — DiagManager
// (include/pic/diag/manager.hpp:24-69): builds the modules named by the deck's
// `[diagnostics] enable` list and fans out sample()/finalize(). The same
// constructor, names and cadences as the reference's; the manager owns the
// writer (AsyncSink) that its modules hand their host work to, and samples on
// the stream the particles were loaded on, so a sample enqueues device work and
// returns without waiting for the GPU. finalize() (or the destructor) waits
// for every pending write.
#ifndef ARC_PIC_DIAG_MANAGER_HPP
#define ARC_PIC_DIAG_MANAGER_HPP

#include "pic/deck.hpp"
#include "pic/diag/em_energy.hpp"
#include "pic/diag/kt.hpp"
#include "pic/diag/module.hpp"
#include "pic/diag/phase_frames.hpp"
#include "pic/diag/phase_video.hpp"
#include "pic/diag/snapshot.hpp"
#include "pic/diag/spectrum.hpp"

#include <cstdio>
#include <memory>
#include <string>
#include <vector>

namespace arc { namespace diag {

class DiagManager {
    std::unique_ptr<AsyncSink> sink_;          // declared first: destroyed after the modules
    std::vector<std::unique_ptr<IDiag>> mods_;
    double bmag_, cost_, sint_, vth_, vr_;
public:
    // pref = output file prefix; outdir = directory for phase_frames and its
    // manifest ("" -> the working directory).
    DiagManager(const Deck& d, const RunParams& rp, const std::string& pref, const std::string& outdir)
        : sink_(std::make_unique<AsyncSink>()) {
        bmag_ = std::sqrt(static_cast<double>(rp.B0[0]) * rp.B0[0] + static_cast<double>(rp.B0[1]) * rp.B0[1] +
                          static_cast<double>(rp.B0[2]) * rp.B0[2]);
        cost_ = bmag_ > 0 ? rp.B0[0] / bmag_ : 1.0;
        sint_ = bmag_ > 0 ? rp.B0[2] / bmag_ : 0.0;
        vth_ = d.species.empty() ? 1.0 : d.species[0].uth[0];
        vr_ = (rp.pump_k0 > 0 && cost_ > 0) ? (rp.pump_w0 / (rp.pump_k0 * cost_)) / vth_ : 0.0;

        for (const std::string& k : d.diag_enable) {
            if (k == "spectrum") mods_.emplace_back(new SpectrumDiag(d));
            else if (k == "kt") mods_.emplace_back(new KTDump(d, pref));
            else if (k == "phase_video") mods_.emplace_back(new PhaseVideo(d, pref));
            else if (k == "snapshot") mods_.emplace_back(new Snapshot(d, pref));
            else if (k == "em_energy") mods_.emplace_back(new EMEnergy(d, pref));
            else if (k == "phase_frames") mods_.emplace_back(new PhaseFrames(d, outdir));
            else std::fprintf(stderr, "DiagManager: unknown diagnostic '%s' (ignored)\n", k.c_str());
        }
    }
    ~DiagManager() {
        try { sink_->flush(); } catch (...) {}
    }

    bool empty() const { return mods_.empty(); }

    void sample(const Fields& f, const Particles& p, const Grid& g, const RunParams& rp, long step, double t) {
        if (mods_.empty()) return;
        DiagFrame fr{f, p, g, rp, step, t, bmag_, cost_, sint_, vth_, vr_, p.stream, sink_.get()};
        for (auto& m : mods_) m->sample(fr);
    }

    void finalize() {
        sink_->flush();
        for (auto& m : mods_) m->finalize();
    }
};

}}  // namespace arc::diag

#endif  // ARC_PIC_DIAG_MANAGER_HPP
