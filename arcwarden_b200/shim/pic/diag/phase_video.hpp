// pic/diag/phase_video.hpp (B200 shim) — PhaseVideo
// (include/pic/diag/phase_video.hpp:14-73): per frame, the f(x, v_par / v_th)
// histogram (256 x 200 float bins) to <pref>vid_phase.bin and the rows E_par,
// E_perp, dB_y to <pref>vid_field.bin; <pref>vid.meta at finalize. The
// reference bins on the GPU and then blocks on cudaMemcpy of the histogram and
// four field rows each frame; here the histogram is counted with integer
// atomics in the same FP32 arithmetic (a private 200 KB copy in each block's
// shared memory, one block per SM), converted to float bins, and copied with
// the rows into a pinned buffer asynchronously; the writer thread forms the
// field rows (in FP64, as the reference) and appends both records.
#ifndef ARC_PIC_DIAG_PHASE_VIDEO_HPP
#define ARC_PIC_DIAG_PHASE_VIDEO_HPP

#include "pic/deck.hpp"
#include "pic/diag/module.hpp"

#include <cstdio>
#include <cstring>
#include <fstream>

namespace arc { namespace diag {

class PhaseVideo : public IDiag {
    static constexpr int   NXB = 256, NVB = 200;
    static constexpr float VLO = -6.0f, VHI = 6.0f;   // v_par / v_th
    int    nx_, stride_;
    double toff_, Lx_, dt_;
    std::string meta_;
    FILE  *vph_ = nullptr, *vfl_ = nullptr;
    int    nframe_ = 0;
    double vr_ = 0.0;
    DeviceArray<unsigned> counts_;
    DeviceArray<float>    dhist_;
    int        sms_ = 148;               // blocks of the counting kernel: one per SM
    AsyncSink* sink_ = nullptr;
public:
    PhaseVideo(const Deck& d, const std::string& pref)
        : nx_(d.nx), stride_(d.rp.nsteps / (d.n_frames > 0 ? d.n_frames : 150) > 0
                                 ? static_cast<int>(d.rp.nsteps / (d.n_frames > 0 ? d.n_frames : 150)) : 1),
          toff_(d.rp.pump_toff), Lx_(d.Lx), dt_(d.rp.dt), meta_(pref + "vid.meta"),
          counts_(static_cast<std::size_t>(NXB) * NVB), dhist_(static_cast<std::size_t>(NXB) * NVB) {
        int dev = 0;
        CUDA_CHECK(cudaGetDevice(&dev));
        CUDA_CHECK(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev));
        CUDA_CHECK(cudaFuncSetAttribute(dev::k_phase_counts_f32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(sizeof(unsigned) * NXB * NVB)));
        vph_ = std::fopen((pref + "vid_phase.bin").c_str(), "wb");
        vfl_ = std::fopen((pref + "vid_field.bin").c_str(), "wb");
    }
    ~PhaseVideo() override {
        try { if (sink_) sink_->flush(); } catch (...) {}
        if (vph_) std::fclose(vph_);
        if (vfl_) std::fclose(vfl_);
    }
    void sample(const DiagFrame& fr) override {
        if (fr.step % stride_ != 0 || !vph_ || !vfl_) return;
        AsyncSink& sink = sink_of(fr);
        sink_ = &sink;
        vr_ = fr.vr;
        const size_t nh = static_cast<size_t>(NXB) * NVB;
        counts_.zero(fr.stream);
        const long np = static_cast<long>(fr.p.n);
        if (np > 0) {
            dev::k_phase_counts_f32<<<sms_, 1024, sizeof(unsigned) * nh, fr.stream>>>(
                fr.p.x.data(), fr.p.ux.data(), fr.p.uz.data(), np, counts_.data(), NXB, NVB, nx_,
                static_cast<float>(fr.cost), static_cast<float>(fr.sint), static_cast<float>(fr.vth), VLO, VHI);
            CUDA_CHECK(cudaPeekAtLastError());
        }
        dev::k_counts_to_float<<<dev::blocks_for(static_cast<long>(nh)), dev::kThreads, 0, fr.stream>>>(
            counts_.data(), dhist_.data(), static_cast<int>(nh));
        CUDA_CHECK(cudaPeekAtLastError());
        // pinned layout: [hist (nh)] [Ex Ey Ez By rows (4 * nx)]
        const size_t row = sizeof(float) * static_cast<size_t>(nx_);
        AsyncSink::Buf b = sink.acquire(sizeof(float) * nh + 4 * row);
        char* h = static_cast<char*>(b.host);
        CUDA_CHECK(cudaMemcpyAsync(h, dhist_.data(), sizeof(float) * nh, cudaMemcpyDeviceToHost, fr.stream));
        char* rows = h + sizeof(float) * nh;
        const bool em = fr.f.Ez.size() > 0;
        CUDA_CHECK(cudaMemcpyAsync(rows, fr.f.Ex.data(), row, cudaMemcpyDeviceToHost, fr.stream));
        CUDA_CHECK(cudaMemcpyAsync(rows + row, fr.f.Ey.data(), row, cudaMemcpyDeviceToHost, fr.stream));
        if (em) {
            CUDA_CHECK(cudaMemcpyAsync(rows + 2 * row, fr.f.Ez.data(), row, cudaMemcpyDeviceToHost, fr.stream));
            CUDA_CHECK(cudaMemcpyAsync(rows + 3 * row, fr.f.By.data(), row, cudaMemcpyDeviceToHost, fr.stream));
        }
        const int nx = nx_;
        const double cost = fr.cost, sint = fr.sint;
        const float b0y = fr.rp.B0[1];
        FILE* vph = vph_;
        FILE* vfl = vfl_;
        sink.submit(b, fr.stream, [=](const void* p) {
            const float* hh = static_cast<const float*>(p);
            const float* ex = hh + nh;
            const float* ey = ex + nx;
            const float* ez = ey + nx;
            const float* by = ez + nx;
            std::fwrite(hh, sizeof(float), nh, vph);
            std::vector<float> frow(3 * static_cast<size_t>(nx));
            for (int i = 0; i < nx; ++i) {
                const double ezi = em ? ez[i] : 0.0, byi = em ? by[i] : 0.0;
                frow[i] = static_cast<float>(ex[i] * cost + ezi * sint);
                frow[nx + i] = ey[i];
                frow[2 * nx + i] = static_cast<float>(byi - b0y);
            }
            std::fwrite(frow.data(), sizeof(float), frow.size(), vfl);
        });
        ++nframe_;
    }
    void finalize() override {
        if (sink_) sink_->flush();
        if (vph_) { std::fclose(vph_); vph_ = nullptr; }
        if (vfl_) { std::fclose(vfl_); vfl_ = nullptr; }
        std::ofstream o(meta_);
        o << "nframe " << nframe_ << "\nnxb " << NXB << "\nnvb " << NVB << "\nnx " << nx_ << "\nLx " << Lx_
          << "\nvlo " << VLO << "\nvhi " << VHI << "\ntoff " << toff_ << "\ndt_frame " << stride_ * dt_
          << "\nvr " << vr_ << "\n";
    }
};

}}  // namespace arc::diag

#endif  // ARC_PIC_DIAG_PHASE_VIDEO_HPP
