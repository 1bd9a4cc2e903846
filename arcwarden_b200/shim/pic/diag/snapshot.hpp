// pic/diag/snapshot.hpp (B200 shim) — Snapshot (include/pic/diag/snapshot.hpp:
// 14-77): at t_snap (or the last step), <pref>fields.csv (x, Epar, Eperp, Ey, dBy,
// dBmag of row 0), <pref>fhist.bin (f(x, v_par / v_th), 512 x 480 float bins over
// every particle) and <pref>fhist.meta. The reference copies x, ux and uz of every
// particle to the host and bins them there in FP64; here the same FP64 binning
// runs on the GPU (integer counts, converted as the reference's float sums leave
// them), and only the 983 KB histogram and six field rows are copied, into a
// pinned buffer, asynchronously; the files are written on the writer thread.
#ifndef ARC_PIC_DIAG_SNAPSHOT_HPP
#define ARC_PIC_DIAG_SNAPSHOT_HPP

#include "pic/deck.hpp"
#include "pic/diag/module.hpp"

#include <cstdio>
#include <cstring>
#include <fstream>

namespace arc { namespace diag {

class Snapshot : public IDiag {
    static constexpr int NXB = 512, NVB = 480;
    static constexpr double VLO = -6.0, VHI = 6.0;   // v_par / v_th
    int    nx_;
    long   snap_step_, last_step_;
    double dx_, Lx_;
    std::string pref_;
    bool   done_ = false;
    AsyncSink* sink_ = nullptr;
    DeviceArray<unsigned> counts_;
    DeviceArray<float>    hist_;
public:
    Snapshot(const Deck& d, const std::string& pref)
        : nx_(d.nx),
          snap_step_(static_cast<long>(std::lround((d.tsnap > 0 ? d.tsnap : d.rp.nsteps * d.rp.dt) / d.rp.dt))),
          last_step_(d.rp.nsteps), dx_(d.Lx / d.nx), Lx_(d.Lx), pref_(pref),
          counts_(static_cast<size_t>(NXB) * NVB), hist_(static_cast<size_t>(NXB) * NVB) {}
    ~Snapshot() override {
        try { if (sink_) sink_->flush(); } catch (...) {}
    }

    void sample(const DiagFrame& fr) override {
        if (done_ || (fr.step < snap_step_ && fr.step < last_step_)) return;
        done_ = true;
        AsyncSink& sink = sink_of(fr);
        sink_ = &sink;
        const Fields& f = fr.f;
        const bool em = f.Ez.size() > 0;
        const Particles& P = fr.p;
        const long Np = static_cast<long>(P.n);
        const size_t nh = static_cast<size_t>(NXB) * NVB;
        counts_.zero(fr.stream);
        if (Np > 0) {
            dev::k_phase_counts_f64<<<dev::blocks_for(Np), dev::kThreads, 0, fr.stream>>>(
                P.x.data(), P.ux.data(), P.uz.data(), Np, counts_.data(), NXB, NVB, dx_, Lx_, fr.cost, fr.sint,
                fr.vth, VLO, VHI);
            CUDA_CHECK(cudaPeekAtLastError());
        }
        dev::k_counts_to_float<<<dev::blocks_for(static_cast<long>(nh)), dev::kThreads, 0, fr.stream>>>(
            counts_.data(), hist_.data(), static_cast<int>(nh));
        CUDA_CHECK(cudaPeekAtLastError());
        // pinned layout: [hist (nh)] [Ex Ey Ez Bx By Bz rows (6 * nx)]
        const size_t row = sizeof(float) * static_cast<size_t>(nx_);
        AsyncSink::Buf b = sink.acquire(sizeof(float) * nh + 6 * row);
        char* h = static_cast<char*>(b.host);
        CUDA_CHECK(cudaMemcpyAsync(h, hist_.data(), sizeof(float) * nh, cudaMemcpyDeviceToHost, fr.stream));
        char* rows = h + sizeof(float) * nh;
        std::memset(rows, 0, 6 * row);
        CUDA_CHECK(cudaMemcpyAsync(rows, f.Ex.data(), row, cudaMemcpyDeviceToHost, fr.stream));
        CUDA_CHECK(cudaMemcpyAsync(rows + row, f.Ey.data(), row, cudaMemcpyDeviceToHost, fr.stream));
        if (em) {
            const float* src[4] = {f.Ez.data(), f.Bx.data(), f.By.data(), f.Bz.data()};
            for (int k = 0; k < 4; ++k)
                CUDA_CHECK(cudaMemcpyAsync(rows + (2 + k) * row, src[k], row, cudaMemcpyDeviceToHost, fr.stream));
        }
        const int nx = nx_;
        const double dx = dx_, Lx = Lx_, cost = fr.cost, sint = fr.sint, t = fr.t, vr = fr.vr;
        const float b0x = fr.rp.B0[0], b0y = fr.rp.B0[1], b0z = fr.rp.B0[2];
        const std::string pref = pref_;
        sink.submit(b, fr.stream, [=](const void* p) {
            const float* hist = static_cast<const float*>(p);
            const float* fex = hist + nh;
            const float* fey = fex + nx;
            const float* fez = fey + nx;
            const float* fbx = fez + nx;
            const float* fby = fbx + nx;
            const float* fbz = fby + nx;
            {
                std::ofstream o(pref + "fields.csv");
                o << "x,Epar,Eperp,Ey,dBy,dBmag\n";
                for (int i = 0; i < nx; ++i) {
                    const double Epar = fex[i] * cost + fez[i] * sint;
                    const double Eperp = fey[i];
                    const double dbx = fbx[i] - b0x, dby = fby[i] - b0y, dbz = fbz[i] - b0z;
                    o << i * dx << ',' << Epar << ',' << Eperp << ',' << fey[i] << ',' << dby << ','
                      << std::sqrt(dbx * dbx + dby * dby + dbz * dbz) << '\n';
                }
            }
            {
                std::ofstream hb(pref + "fhist.bin", std::ios::binary);
                hb.write(reinterpret_cast<const char*>(hist), nh * sizeof(float));
            }
            {
                std::ofstream m(pref + "fhist.meta");
                m << "nxb " << NXB << "\nnvb " << NVB << "\nLx " << Lx << "\nvlo " << VLO << "\nvhi " << VHI
                  << "\nvr " << vr << "\ntsnap " << t << "\n";
            }
            std::printf("  [snapshot] wrote %sfields.csv + %sfhist.bin at t=%.1f (%dx%d over %ld particles)\n",
                        pref.c_str(), pref.c_str(), t, NXB, NVB, Np);
        });
    }
    void finalize() override {
        if (sink_) sink_->flush();
    }
};

}}  // namespace arc::diag

#endif  // ARC_PIC_DIAG_SNAPSHOT_HPP
