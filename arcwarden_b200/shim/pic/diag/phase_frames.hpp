// pic/diag/phase_frames.hpp (B200 shim) — PhaseFrames
// (include/pic/diag/phase_frames.hpp:19-65): (x, vx) phase-space CSV frames of a
// fixed random sample of at most 100k particles, plus a manifest. Cadence, sample
// (std::mt19937 seeded 12345, shuffle, first 100k, sorted), file names and the
// CSV text are the reference's. The reference copies x and ux of every particle
// to the host per frame; here the sample's indices live on the GPU, a gather
// kernel writes the sampled (x, ux) pairs and only those (800 KB at most) are
// copied, asynchronously, to a pinned buffer; the CSV is written on the
// diagnostics writer thread, its text made with std::to_chars (the bytes that
// the reference's ostream writes).
#ifndef ARC_PIC_DIAG_PHASE_FRAMES_HPP
#define ARC_PIC_DIAG_PHASE_FRAMES_HPP

#include "pic/deck.hpp"
#include "pic/diag/csv_text.hpp"
#include "pic/diag/module.hpp"

#include <algorithm>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <memory>
#include <numeric>
#include <random>
#include <thread>

namespace arc { namespace diag {

class PhaseFrames : public IDiag {
    static constexpr int CAP = 100000;
    long   stride_;
    double dt_;
    std::string dir_;
    std::shared_ptr<std::ofstream> man_;
    int    frame_ = 0;
    bool   inited_ = false;
    int    m_ = 0;                 // sampled particles
    bool   all_ = false;           // every particle sampled, in index order
    DeviceArray<int>   idx_;       // the sample's indices (when not all_)
    DeviceArray<float> out_;       // gathered [x(m), ux(m)]
    AsyncSink* sink_ = nullptr;
public:
    PhaseFrames(const Deck& d, const std::string& outdir)
        : stride_(d.dump_every > 0 ? d.dump_every : (d.rp.nsteps / 100 > 0 ? d.rp.nsteps / 100 : 1)),
          dt_(d.rp.dt), dir_(outdir.empty() ? "." : outdir),
          man_(std::make_shared<std::ofstream>()) {
        std::filesystem::create_directories(dir_);
        man_->open(dir_ + "/manifest.csv");
        if (*man_) *man_ << "frame,step,time,file\n";
    }
    ~PhaseFrames() override {
        try { if (sink_) sink_->flush(); } catch (...) {}
    }
    void sample(const DiagFrame& fr) override {
        if (fr.step % stride_ != 0) return;
        AsyncSink& sink = sink_of(fr);
        sink_ = &sink;
        const int N = static_cast<int>(fr.p.n);
        if (!inited_) {
            all_ = N <= CAP;
            m_ = all_ ? N : CAP;
            if (!all_) {
                std::vector<int> idx(N);
                std::iota(idx.begin(), idx.end(), 0);
                std::mt19937 rng(12345);
                std::shuffle(idx.begin(), idx.end(), rng);
                idx.resize(CAP);
                std::sort(idx.begin(), idx.end());
                idx_ = DeviceArray<int>(CAP);
                out_ = DeviceArray<float>(2 * static_cast<size_t>(CAP));
                CUDA_CHECK(cudaMemcpy(idx_.data(), idx.data(), sizeof(int) * CAP, cudaMemcpyHostToDevice));
            }
            inited_ = true;
        }
        const int m = m_;
        const size_t row = sizeof(float) * static_cast<size_t>(m);
        AsyncSink::Buf b = sink.acquire(2 * row);
        if (m > 0) {
            if (all_) {
                CUDA_CHECK(cudaMemcpyAsync(b.host, fr.p.x.data(), row, cudaMemcpyDeviceToHost, fr.stream));
                CUDA_CHECK(cudaMemcpyAsync(static_cast<char*>(b.host) + row, fr.p.ux.data(), row,
                                           cudaMemcpyDeviceToHost, fr.stream));
            } else {
                dev::k_gather_x_ux<<<dev::blocks_for(m), dev::kThreads, 0, fr.stream>>>(
                    fr.p.x.data(), fr.p.ux.data(), idx_.data(), m, out_.data());
                CUDA_CHECK(cudaPeekAtLastError());
                CUDA_CHECK(cudaMemcpyAsync(b.host, out_.data(), 2 * row, cudaMemcpyDeviceToHost, fr.stream));
            }
        }
        char name[64];
        std::snprintf(name, sizeof name, "frame_%04d.csv", frame_);
        const std::string path = dir_ + "/" + name, file = name;
        const int nx = fr.g.nx;
        const double dx = fr.g.dx;
        const long step = fr.step;
        const double t = fr.t;
        const int frame = frame_;
        std::shared_ptr<std::ofstream> man = man_;
        sink.submit(b, fr.stream, [=](const void* p) {
            const float* x = static_cast<const float*>(p);
            const float* vx = x + m;
            write_frame(path, x, vx, m, nx, dx);
            if (*man) {
                *man << frame << ',' << step << ',' << t << ',' << file << '\n';
                man->flush();
            }
        });
        ++frame_;
    }
    void finalize() override {
        if (sink_) sink_->flush();
    }

    // frame_%04d.csv: "x,vx" then one row per sampled particle, x wrapped into
    // [0, nx) in FP32 and scaled by dx, the text of `o << x * dx << ',' << vx`;
    // rows are formatted in up to four parallel slices and written in order.
    static void write_frame(const std::string& path, const float* x, const float* vx, int m, int nx, double dx) {
        const int nslice = m < 4096 ? 1 : 4;
        std::vector<std::vector<char>> text(nslice);
        auto fill = [&](int s) {
            const int lo = static_cast<int>(static_cast<long>(m) * s / nslice);
            const int hi = static_cast<int>(static_cast<long>(m) * (s + 1) / nslice);
            std::vector<char>& out = text[s];
            out.resize(static_cast<size_t>(hi - lo) * kRow2Max);
            char* q = out.data();
            for (int k = lo; k < hi; ++k) {
                float xd = x[k];
                if (xd < 0.0f) xd += nx;
                else if (xd >= nx) xd -= nx;
                q = put_row2(q, xd * dx, vx[k]);
            }
            out.resize(static_cast<size_t>(q - out.data()));
        };
        std::vector<std::thread> th;
        for (int s = 1; s < nslice; ++s) th.emplace_back(fill, s);
        fill(0);
        for (std::thread& t : th) t.join();
        FILE* f = std::fopen(path.c_str(), "wb");
        if (!f) return;
        std::fputs("x,vx\n", f);
        for (const std::vector<char>& v : text) std::fwrite(v.data(), 1, v.size(), f);
        std::fclose(f);
    }
};

}}  // namespace arc::diag

#endif  // ARC_PIC_DIAG_PHASE_FRAMES_HPP
