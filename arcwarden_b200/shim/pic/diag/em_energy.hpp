// pic/diag/em_energy.hpp (B200 shim) — EMEnergy
// (include/pic/diag/em_energy.hpp:13-41): Darwin field energies
// 0.5 dx dy sum(component^2) of E, B and E_T to <pref>emenergy.csv every
// nsteps/40 steps, and the final line at finalize. The reference synchronises
// and copies all nine grids to the host per sample; here one FP64 reduction
// kernel (fixed order) sums the three groups on the GPU and 24 bytes are
// copied into a pinned buffer asynchronously; the writer thread writes the row.
#ifndef ARC_PIC_DIAG_EM_ENERGY_HPP
#define ARC_PIC_DIAG_EM_ENERGY_HPP

#include "pic/deck.hpp"
#include "pic/diag/module.hpp"

#include <fstream>
#include <memory>

namespace arc { namespace diag {

class EMEnergy : public IDiag {
    struct Last {
        double eE = 0, eB = 0, eT = 0;
    };
    long   every_;
    std::shared_ptr<std::ofstream> csv_;
    std::shared_ptr<Last> last_;      // written by the writer thread, read after flush
    DeviceArray<double> red_;
    AsyncSink* sink_ = nullptr;
public:
    EMEnergy(const Deck& d, const std::string& pref)
        : every_(d.rp.nsteps / 40 > 0 ? d.rp.nsteps / 40 : 1), csv_(std::make_shared<std::ofstream>()),
          last_(std::make_shared<Last>()), red_(3 * dev::kBlocks + 3) {
        csv_->open(pref + "emenergy.csv");
        if (*csv_) *csv_ << "step,time,E_total,B,E_T\n";
    }
    ~EMEnergy() override {
        try { if (sink_) sink_->flush(); } catch (...) {}
    }
    void sample(const DiagFrame& fr) override {
        if (fr.step % every_ != 0 || fr.f.Ez.size() == 0) return;
        AsyncSink& sink = sink_of(fr);
        sink_ = &sink;
        const Fields& f = fr.f;
        dev::SqTerms t{};
        const float* a[9] = {f.Ex.data(), f.Ey.data(), f.Ez.data(), f.Bx.data(), f.By.data(),
                             f.Bz.data(), f.ETx.data(), f.ETy.data(), f.ETz.data()};
        const size_t sz[9] = {f.Ex.size(), f.Ey.size(), f.Ez.size(), f.Bx.size(), f.By.size(),
                              f.Bz.size(), f.ETx.size(), f.ETy.size(), f.ETz.size()};
        const long n = static_cast<long>(f.Ex.size());
        for (int k = 0; k < 9; ++k) {
            if (sz[k] == 0) continue;
            if (static_cast<long>(sz[k]) != n) throw CudaError("EMEnergy: field arrays of different sizes");
            t.a[t.count] = a[k];
            t.off[t.count] = 0.0f;
            t.group[t.count] = k / 3;
            ++t.count;
        }
        dev::sq_sums(t, n, red_.data(), red_.data() + 3 * dev::kBlocks, fr.stream);
        AsyncSink::Buf b = sink.acquire(3 * sizeof(double));
        CUDA_CHECK(cudaMemcpyAsync(b.host, red_.data() + 3 * dev::kBlocks, 3 * sizeof(double),
                                   cudaMemcpyDeviceToHost, fr.stream));
        const double cell = 0.5 * fr.g.dx * fr.g.dy;
        const long step = fr.step;
        const double time = fr.t;
        std::shared_ptr<std::ofstream> csv = csv_;
        std::shared_ptr<Last> last = last_;
        sink.submit(b, fr.stream, [=](const void* p) {
            const double* s = static_cast<const double*>(p);
            last->eE = cell * s[0];
            last->eB = cell * s[1];
            last->eT = cell * s[2];
            if (*csv) *csv << step << ',' << time << ',' << last->eE << ',' << last->eB << ',' << last->eT << '\n';
        });
    }
    void finalize() override {
        if (sink_) sink_->flush();
        const double eE = last_->eE, eB = last_->eB, eT = last_->eT;
        std::printf("  final field energy: electric(E_total)=%.4e  magnetic=%.4e (%.2e of E)"
                    "  transverse-E=%.4e (%.2e of E)\n",
                    eE, eB, eE > 0 ? eB / eE : 0.0, eT, eE > 0 ? eT / eE : 0.0);
    }
};

}}  // namespace arc::diag

#endif  // ARC_PIC_DIAG_EM_ENERGY_HPP
