// pic/pump.hpp (B200 shim) — add_background_b0 / add_pump_field
// (include/pic/pump.hpp:59-79) on libarcb200.
#ifndef ARC_PIC_PUMP_HPP
#define ARC_PIC_PUMP_HPP

#include "pic/config.hpp"
#include "pic/fields.hpp"
#include "pic/grid.hpp"

#include "../arcb200_shim.hpp"

namespace arc {

// B += B0 on the grid.
inline void add_background_b0(Fields& fld, const Grid& g, const RunParams& rp, cudaStream_t s) {
    aw_ctx* c = shim::prepare(g, rp, true, s);
    shim::bind_fields(c, fld);
    shim::check(aw_add_b0(c), "add_b0");
}

// E += the external pump at time t (nothing when the pump is off or t >= t_off).
inline void add_pump_field(Fields& fld, const Grid& g, const RunParams& rp, double t, cudaStream_t s) {
    if (!rp.pump || t >= rp.pump_toff) return;
    aw_ctx* c = shim::prepare(g, rp, true, s);
    shim::bind_fields(c, fld);
    shim::check(aw_add_pump(c, t), "add_pump");
}

}  // namespace arc

#endif  // ARC_PIC_PUMP_HPP
