// pic/diag/csv_text.hpp (B200 shim) — the text of a number as a default
// std::ostream writes it (`o << v`: the %g form with 6 significant digits), made
// with std::to_chars, which is specified to give printf's %.6g in the C locale,
// so the shim's CSV files hold the same bytes as the reference's ostream output
// at a fraction of the cost. Plain C++ (no CUDA), so it can be checked on the host.
#ifndef ARC_PIC_DIAG_CSV_TEXT_HPP
#define ARC_PIC_DIAG_CSV_TEXT_HPP

#include <charconv>
#include <cstddef>

namespace arc { namespace diag {

// Writes v at p (at most 32 bytes) and returns the end of the text.
inline char* put_g6(char* p, double v) {
    return std::to_chars(p, p + 32, v, std::chars_format::general, 6).ptr;
}

// "<a>,<b>\n" as `o << a << ',' << b << '\n'` writes it, for a double a and a
// float b (ostream prints a float through its double value).
inline char* put_row2(char* p, double a, float b) {
    p = put_g6(p, a);
    *p++ = ',';
    p = put_g6(p, static_cast<double>(b));
    *p++ = '\n';
    return p;
}

constexpr std::size_t kRow2Max = 2 * 32 + 2;   // bytes one put_row2 may write

}}  // namespace arc::diag

#endif  // ARC_PIC_DIAG_CSV_TEXT_HPP
