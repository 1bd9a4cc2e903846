// pic/solver_darwin.hpp (B200 shim) — DarwinSpectralSolver
// (include/pic/solver_darwin.hpp:146-264) on libarcb200.
#ifndef ARC_PIC_SOLVER_DARWIN_HPP
#define ARC_PIC_SOLVER_DARWIN_HPP

#include "pic/config.hpp"
#include "pic/fields.hpp"
#include "pic/sources.hpp"
#include "pic/spectral.hpp"

#include "../arcb200_shim.hpp"

namespace arc {

class DarwinSpectralSolver {
public:
    // rho, J -> E (= E_L) into Ex, Ey, Ez = 0, and B.
    void solve(const Sources& src, Fields& fld, SpectralEngine& eng, const RunParams& rp, cudaStream_t s) const {
        call(src, fld, eng.grid(), rp, s, aw_solve_darwin, "solve_darwin");
    }
    // rho, J -> E_L into ELx, ELy, and B.
    void solve_el_b(const Sources& src, Fields& fld, SpectralEngine& eng, const RunParams& rp,
                    cudaStream_t s) const {
        call(src, fld, eng.grid(), rp, s, aw_solve_darwin_el_b, "solve_darwin_el_b");
    }
    // dcu, amu -> E_T into ETx, ETy, ETz (one shot, resummed Green's function).
    void solve_et(const Sources& src, Fields& fld, SpectralEngine& eng, const RunParams& rp,
                  cudaStream_t s) const {
        call(src, fld, eng.grid(), rp, s, aw_solve_darwin_et, "solve_darwin_et");
    }
    // E = E_L + et_scale * E_T.
    void form_e(Fields& fld, float et_scale, cudaStream_t s) const {
        const Grid g = grid_of(fld);
        aw_ctx* c = shim::prepare(g, RunParams{}, true, s);
        shim::bind_fields(c, fld);
        shim::check(aw_form_e(c, et_scale), "form_e");
    }
    void form_el(Fields& fld, cudaStream_t s) const { form_e(fld, 0.0f, s); }
    void form_etotal(Fields& fld, cudaStream_t s) const { form_e(fld, 1.0f, s); }

private:
    static void call(const Sources& src, Fields& fld, const Grid& g, const RunParams& rp, cudaStream_t s,
                     int (*op)(aw_ctx*), const char* what) {
        aw_ctx* c = shim::prepare(g, rp, true, s);
        shim::bind_sources(c, const_cast<Sources&>(src));
        shim::bind_fields(c, fld);
        shim::check(op(c), what);
    }
    // form_e names no grid: use the grid of the last call when its size
    // matches the fields (the usual case), else any grid with as many cells
    // (the combine is elementwise).
    static Grid grid_of(const Fields& fld) {
        const int n = static_cast<int>(fld.Ex.size());
        const Grid& g = shim::last_grid();
        if (g.real_size() == n) return g;
        return Grid(n, 1, static_cast<double>(n), 1.0);
    }
};

}  // namespace arc

#endif  // ARC_PIC_SOLVER_DARWIN_HPP
