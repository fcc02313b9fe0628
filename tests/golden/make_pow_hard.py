"""Writes tests/golden/pow_quarter_hard.npz: inputs x of the RK45 controller's
pow(x, 0.25) whose exact fourth root lies within 2^-14 ulp of a rounding tie,
together with glibc's pow(x, 0.25) on the machine that ran this script.

These are the inputs on which a pow that is not correctly rounded can round
either way, so they are where a restatement of glibc's pow
(gr-ray-tracer_b200/csrc/grt_pow_quarter.cuh) is tested hardest.  The exact
root comes from libquadmath's powq (113 bits); x is drawn log-uniformly over
the controller's unclamped range [1.5e-8, 2e4] and over all normal doubles.

Usage: python make_pow_hard.py   (needs g++ with libquadmath)
"""

import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

SRC = r"""
#include <quadmath.h>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <omp.h>
static inline uint64_t xr(uint64_t* s) { *s ^= *s << 13; *s ^= *s >> 7; *s ^= *s << 17; return *s; }
int main(int argc, char** argv) {
    const long n = atol(argv[1]);
    const double lo = atof(argv[2]), hi = atof(argv[3]);
    const double tol = ldexp(1.0, -14);
    FILE* f = fopen(argv[4], "wb");
    long kept = 0;
    #pragma omp parallel
    {
        uint64_t s = 0x2545F4914F6CDD1Dull;
        s ^= 0x9E3779B97F4A7C15ull * (uint64_t)(omp_get_thread_num() + 1);
        #pragma omp for
        for (long j = 0; j < n; ++j) {
            const double u = (xr(&s) >> 11) * 0x1p-53;
            const double x = exp(log(lo) + u * (log(hi) - log(lo)));
            const __float128 v = powq((__float128)x, 0.25Q);
            const double d = (double)v;
            const __float128 ulp = (__float128)ldexp(1.0, ilogb(d) - 52);
            const double frac = (double)(fabsq(v - (__float128)d) / ulp);  // in [0, 0.5]
            if (0.5 - frac < tol) {
                const double y = pow(x, 0.25);
                #pragma omp critical
                { fwrite(&x, 8, 1, f); fwrite(&y, 8, 1, f); ++kept; }
            }
        }
    }
    fclose(f);
    printf("%ld\n", kept);
    return 0;
}
"""


def run(n, lo, hi, tmp):
    exe = tmp / "hard"
    out = tmp / f"out_{lo}_{hi}.bin"
    subprocess.run([str(exe), str(n), repr(lo), repr(hi), str(out)], check=True, capture_output=True, text=True)
    a = np.fromfile(out, dtype=np.float64).reshape(-1, 2)
    return a[np.argsort(a[:, 0], kind="stable")]


def main():
    with tempfile.TemporaryDirectory() as d:
        tmp = Path(d)
        (tmp / "hard.cpp").write_text(SRC)
        subprocess.run(["g++", "-O2", "-fopenmp", "-ffp-contract=off", str(tmp / "hard.cpp"), "-o", str(tmp / "hard"),
                        "-lquadmath"], check=True)
        ctrl = run(200_000_000, 1.5e-8, 2e4, tmp)
        wide = run(50_000_000, 2.3e-308, 1.7e308, tmp)
    np.savez_compressed(HERE / "pow_quarter_hard.npz", x_controller=ctrl[:, 0], pow_controller=ctrl[:, 1],
                        x_wide=wide[:, 0], pow_wide=wide[:, 1])
    print(f"wrote {len(ctrl)} + {len(wide)} tie-near inputs")


if __name__ == "__main__":
    main()
