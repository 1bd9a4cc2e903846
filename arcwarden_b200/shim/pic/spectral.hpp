// pic/spectral.hpp (B200 shim) — SpectralEngine (include/pic/spectral.hpp:
// 106-149) on libarcb200's cuFFT plans, with the reference's workspace and
// form-factor types so code that names them compiles unchanged.
#ifndef ARC_PIC_SPECTRAL_HPP
#define ARC_PIC_SPECTRAL_HPP

#include "pic/cuda_utils.hpp"
#include "pic/device_array.hpp"
#include "pic/grid.hpp"

#include "../arcb200_shim.hpp"

#include <cufft.h>

namespace arc {

// k-space buffers by name (allocated for API compatibility; the library keeps
// its own batched k-space planes).
struct SpectralWorkspace {
    DeviceArray<cufftComplex> rho_k, phi_k, Ex_k, Ey_k;
    DeviceArray<cufftComplex> Jx_k, Jy_k, Jz_k, Bx_k, By_k, Bz_k;
    DeviceArray<cufftComplex> ETx_k, ETy_k, ETz_k, dcux_k, dcuy_k, dcuz_k;
    DeviceArray<cufftComplex> amu0_k, amu1_k, amu2_k, amu3_k;

    SpectralWorkspace() = default;
    explicit SpectralWorkspace(int nk) : rho_k(nk), phi_k(nk), Ex_k(nk), Ey_k(nk) {}

    void allocate_em(int nk) {
        DeviceArray<cufftComplex>* em[] = {&Jx_k, &Jy_k, &Jz_k, &Bx_k, &By_k, &Bz_k, &ETx_k, &ETy_k,
                                           &ETz_k, &dcux_k, &dcuy_k, &dcuz_k, &amu0_k, &amu1_k, &amu2_k, &amu3_k};
        for (auto* a : em) *a = DeviceArray<cufftComplex>(nk);
    }
};

// Green's functions of the solves (eps0, c, n0 as in RunParams).
struct SpectralFormFactor {
    double eps0 = 1.0;
    double c = 1.0;
    double n0 = 1.0;
    __host__ __device__ double smoothing(double) const { return 1.0; }
    __host__ __device__ double green(double k2) const { return k2 > 0.0 ? 1.0 / (eps0 * k2) : 0.0; }
    __host__ __device__ double green_t(double k2) const { return k2 > 0.0 ? 1.0 / (eps0 * c * c * k2) : 0.0; }
    __host__ __device__ double green_et(double k2) const {
        return k2 > 0.0 ? 1.0 / (eps0 * c * c * k2 + n0) : 0.0;
    }
};

class SpectralEngine {
public:
    explicit SpectralEngine(const Grid& g, int batch = 1) : grid_(g), kgrid_(g), ws_(kgrid_.complex_size()) {
        (void)batch;
    }

    // Forward R2C, unnormalised: real [ny][nx] -> half-complex [ny][nx/2+1].
    void r2c(const float* in, cufftComplex* out, cudaStream_t s) const {
        aw_ctx* c = ctx(s);
        shim::check(aw_fft_r2c(c, in, out), "fft_r2c");
    }
    // Inverse C2R normalised by 1/(nx ny); consumes its input like cuFFT.
    void c2r(cufftComplex* in, float* out, cudaStream_t s) const {
        aw_ctx* c = ctx(s);
        shim::check(aw_fft_c2r(c, in, out), "fft_c2r");
    }

    void enable_em() { ws_.allocate_em(kgrid_.complex_size()); }

    SpectralWorkspace&        ws() { return ws_; }
    const SpectralWorkspace&  ws() const { return ws_; }
    const Grid&               grid() const { return grid_; }
    const KGrid&              kgrid() const { return kgrid_; }
    const SpectralFormFactor& form_factor() const { return ff_; }

private:
    aw_ctx* ctx(cudaStream_t s) const {
        aw_ctx* c = shim::context(grid_, AW_MODEL_DARWIN);
        shim::check(aw_set_stream(c, s), "set_stream");
        return c;
    }
    Grid grid_;
    KGrid kgrid_;
    SpectralWorkspace ws_;
    SpectralFormFactor ff_;
};

}  // namespace arc

#endif  // ARC_PIC_SPECTRAL_HPP
