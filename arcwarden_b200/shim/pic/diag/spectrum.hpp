// pic/diag/spectrum.hpp (B200 shim) — SpectrumDiag
// (include/pic/diag/spectrum.hpp:11-48): every nsteps/40 steps a console line with
// |E_M|^2, |E_2M|^2, |E_3M|^2, the band power and dB_rms/B0. The reference copies
// row 0 of Ex and, for Darwin, all of Bx, By, Bz to the host and sums there; here
// the sum of |B - B0|^2 over the grid is an FP64 reduction on the GPU (fixed
// order) and only the row and that one number are copied, asynchronously; the
// mode powers (direct DFTs of the row) and the line come from the writer thread.
#ifndef ARC_PIC_DIAG_SPECTRUM_HPP
#define ARC_PIC_DIAG_SPECTRUM_HPP

#include "pic/deck.hpp"
#include "pic/diag/module.hpp"

#include <cstring>

namespace arc { namespace diag {

class SpectrumDiag : public IDiag {
    int  nx_, M_, blo_, bhi_;
    long every_;
    DeviceArray<double> red_;        // block partials + 3 sums
    AsyncSink* sink_ = nullptr;
public:
    explicit SpectrumDiag(const Deck& d)
        : nx_(d.nx), M_(d.pump_M), blo_(d.band_lo), bhi_(d.band_hi),
          every_(d.rp.nsteps / 40 > 0 ? d.rp.nsteps / 40 : 1), red_(3 * dev::kBlocks + 3) {}
    ~SpectrumDiag() override {
        try { if (sink_) sink_->flush(); } catch (...) {}
    }

    void sample(const DiagFrame& fr) override {
        if (fr.step % every_ != 0) return;
        AsyncSink& sink = sink_of(fr);
        sink_ = &sink;
        const long N = fr.g.real_size();
        const bool mag = fr.f.Bx.size() > 0;
        const size_t row = sizeof(float) * static_cast<size_t>(nx_);
        AsyncSink::Buf b = sink.acquire(row + sizeof(double));
        CUDA_CHECK(cudaMemcpyAsync(b.host, fr.f.Ex.data(), row, cudaMemcpyDeviceToHost, fr.stream));
        if (mag) {
            dev::SqTerms t{};
            const float* a[3] = {fr.f.Bx.data(), fr.f.By.data(), fr.f.Bz.data()};
            for (int k = 0; k < 3; ++k) {
                t.a[k] = a[k];
                t.off[k] = fr.rp.B0[k];
                t.group[k] = 0;
            }
            t.count = 3;
            dev::sq_sums(t, N, red_.data(), red_.data() + 3 * dev::kBlocks, fr.stream);
            CUDA_CHECK(cudaMemcpyAsync(static_cast<char*>(b.host) + row, red_.data() + 3 * dev::kBlocks,
                                       sizeof(double), cudaMemcpyDeviceToHost, fr.stream));
        }
        const int nx = nx_, M = M_, blo = blo_, bhi = bhi_;
        const double t = fr.t, bmag = fr.bmag;
        sink.submit(b, fr.stream, [=](const void* p) {
            const float* exr = static_cast<const float*>(p);
            const std::vector<float> ex(exr, exr + nx);
            const double pM = mode_power(ex, nx, M > 0 ? M : 1);
            const double p2M = mode_power(ex, nx, M > 0 ? 2 * M : 2);
            const double p3M = mode_power(ex, nx, M > 0 ? 3 * M : 3);
            double pB = 0;
            for (int m = blo; m <= bhi; ++m) pB += mode_power(ex, nx, m);
            double dBB0 = 0.0;
            if (mag) {
                double db;
                std::memcpy(&db, static_cast<const char*>(p) + row, sizeof(double));
                dBB0 = std::sqrt(db / N) / (bmag > 0 ? bmag : 1.0);
            }
            std::printf("t=%7.1f  |E_M|2=%.3e |E_2M|2=%.3e |E_3M|2=%.3e  band[%d-%d]=%.3e  dB/B0=%.4f\n", t, pM,
                        p2M, p3M, blo, bhi, pB, dBB0);
        });
    }
    void finalize() override {
        if (sink_) sink_->flush();
    }
};

}}  // namespace arc::diag

#endif  // ARC_PIC_DIAG_SPECTRUM_HPP
