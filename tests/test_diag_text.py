"""The shim's CSV number text (arcwarden_b200/shim/pic/diag/csv_text.hpp, used by
the phase-frame writer) is byte-for-byte what a default std::ostream writes for
the same values, as the reference's PhaseFrames does
(include/pic/diag/phase_frames.hpp:55-59): checked on the host over random bit
patterns (every finite, subnormal, infinite and NaN class) and edge values."""
import shutil
import subprocess

import pytest

from conftest import ROOT

PROGRAM = r"""
#include "pic/diag/csv_text.hpp"
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <random>
#include <sstream>
#include <string>

int main() {
    std::mt19937_64 rng(20260628);
    long n = 0, bad = 0;
    auto check = [&](double a, float b) {
        std::ostringstream o;
        o << a << ',' << b << '\n';
        char buf[arc::diag::kRow2Max];
        char* e = arc::diag::put_row2(buf, a, b);
        ++n;
        if (std::string(buf, e) != o.str()) {
            if (bad < 5) std::printf("mismatch: [%s] vs [%s]\n", std::string(buf, e).c_str(), o.str().c_str());
            ++bad;
        }
    };
    for (int i = 0; i < 400000; ++i) {
        const uint64_t u = rng();
        float f;
        double d;
        const uint32_t u32 = static_cast<uint32_t>(u);
        std::memcpy(&f, &u32, 4);
        std::memcpy(&d, &u, 8);
        check(d, f);
        check(static_cast<double>(f) * 0.25, f);   // the frame's x * dx form
    }
    const float edge[] = {0.0f, -0.0f, 1.0f, -1.0f, 1e-45f, 1.17549435e-38f, 3.4028235e38f,
                          std::numeric_limits<float>::infinity(), -std::numeric_limits<float>::infinity(),
                          std::numeric_limits<float>::quiet_NaN(), 999999.5f, 9999995.0f, 0.0001f, 0.00001f,
                          123456.7f, 1234567.0f, 0.1f, 2048.0f};
    for (float a : edge)
        for (float b : edge) check(static_cast<double>(a) * 0.5, b);
    std::printf("checked %ld rows, %ld mismatches\n", n, bad);
    return bad == 0 ? 0 : 1;
}
"""


def test_csv_text_is_the_ostream_text(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    src = tmp_path / "t.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "t"
    subprocess.run([gxx, "-std=c++20", "-O2", "-I", str(ROOT / "arcwarden_b200" / "shim"), str(src), "-o",
                    str(exe)], check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout
    assert "0 mismatches" in r.stdout
