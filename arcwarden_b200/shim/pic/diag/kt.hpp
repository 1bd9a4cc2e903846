// pic/diag/kt.hpp (B200 shim) — KTDump (include/pic/diag/kt.hpp:14-47): row 0 of
// the longitudinal field ELx appended to <pref>kt.bin every kt_stride steps, and
// <pref>kt.meta at finalize. The reference synchronises the device and copies the
// row with a blocking cudaMemcpy each sample; here the row is copied into a
// pinned buffer asynchronously and appended by the writer thread.
#ifndef ARC_PIC_DIAG_KT_HPP
#define ARC_PIC_DIAG_KT_HPP

#include "pic/deck.hpp"
#include "pic/diag/module.hpp"

#include <cstdio>
#include <fstream>

namespace arc { namespace diag {

class KTDump : public IDiag {
    int    nx_, stride_, M_, blo_, bhi_;
    double w0_, k0_, toff_, Lx_, dt_;
    std::string meta_;
    FILE*  fp_ = nullptr;
    int    nsamp_ = 0;
    AsyncSink* sink_ = nullptr;
public:
    KTDump(const Deck& d, const std::string& pref)
        : nx_(d.nx), stride_(d.kt_stride > 0 ? d.kt_stride : 5), M_(d.pump_M), blo_(d.band_lo),
          bhi_(d.band_hi), w0_(d.rp.pump_w0), k0_(d.rp.pump_k0), toff_(d.rp.pump_toff), Lx_(d.Lx), dt_(d.rp.dt),
          meta_(pref + "kt.meta") {
        fp_ = std::fopen((pref + "kt.bin").c_str(), "wb");
    }
    ~KTDump() override {
        try { if (sink_) sink_->flush(); } catch (...) {}
        if (fp_) std::fclose(fp_);
    }
    void sample(const DiagFrame& fr) override {
        if (fr.step % stride_ != 0 || !fp_ || fr.f.ELx.size() == 0) return;
        AsyncSink& sink = sink_of(fr);
        sink_ = &sink;
        const size_t row = sizeof(float) * static_cast<size_t>(nx_);
        AsyncSink::Buf b = sink.acquire(row);
        CUDA_CHECK(cudaMemcpyAsync(b.host, fr.f.ELx.data(), row, cudaMemcpyDeviceToHost, fr.stream));
        FILE* fp = fp_;
        const int nx = nx_;
        sink.submit(b, fr.stream, [=](const void* p) { std::fwrite(p, sizeof(float), nx, fp); });
        ++nsamp_;
    }
    void finalize() override {
        if (sink_) sink_->flush();
        if (fp_) { std::fclose(fp_); fp_ = nullptr; }
        std::ofstream o(meta_);
        o << "nx " << nx_ << "\nnsamp " << nsamp_ << "\ndt_sample " << stride_ * dt_ << "\ntoff " << toff_
          << "\nLx " << Lx_ << "\nM " << M_ << "\nw0 " << w0_ << "\nband_lo " << blo_ << "\nband_hi " << bhi_
          << "\nvphx " << (k0_ > 0 ? w0_ / k0_ : 0.0) << "\n";
    }
};

}}  // namespace arc::diag

#endif  // ARC_PIC_DIAG_KT_HPP
