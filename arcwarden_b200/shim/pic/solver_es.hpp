// pic/solver_es.hpp (B200 shim) — ElectrostaticSpectralSolver
// (include/pic/solver_es.hpp:80-107) on libarcb200: rho -> Ex, Ey.
#ifndef ARC_PIC_SOLVER_ES_HPP
#define ARC_PIC_SOLVER_ES_HPP

#include "pic/config.hpp"
#include "pic/fields.hpp"
#include "pic/sources.hpp"
#include "pic/spectral.hpp"

#include "../arcb200_shim.hpp"

namespace arc {

class ElectrostaticSpectralSolver {
public:
    void solve(const Sources& src, Fields& fld, SpectralEngine& eng, const RunParams& rp, cudaStream_t s) const {
        aw_ctx* c = shim::prepare(eng.grid(), rp, true, s);
        shim::bind_sources(c, const_cast<Sources&>(src));
        shim::bind_fields(c, fld);
        shim::check(aw_solve_es(c), "solve_es");
    }
};

}  // namespace arc

#endif  // ARC_PIC_SOLVER_ES_HPP
