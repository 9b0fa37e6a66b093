#!/usr/bin/env python
"""Writes tests/golden/seed_seq_rhs.json: right-hand sides drawn as the reference's time loop draws
them (``src/solver/time_loop.cpp:31-43``: ``std::mt19937_64`` seeded by
``std::seed_seq{seed, step, corrector, 0x5eed}``, ``std::uniform_real_distribution<double>(-1, 1)``),
produced by libstdc++ itself through a ten-line C++ program compiled here with g++.

Run where g++ is: python tests/golden/make_seed_seq_golden.py
"""
from __future__ import annotations

import json
import os
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))

CASES = [(12345, 0, 0), (12345, 0, 1), (12345, 7, 2), (1, 31, 15), (4294967295, 1000, 0)]
N = 500

SRC = r"""
#include <cstdio>
#include <cstdlib>
#include <random>
int main(int argc, char** argv) {
    unsigned seed = std::strtoul(argv[1], 0, 10), step = std::atoi(argv[2]), corr = std::atoi(argv[3]);
    int n = std::atoi(argv[4]);
    std::seed_seq seq{seed, step, corr, 0x5eedu};
    std::mt19937_64 gen(seq);
    std::uniform_real_distribution<double> dist(-1.0, 1.0);
    for (int i = 0; i < n; ++i) std::printf("%a\n", dist(gen));
    return 0;
}
"""


def main():
    with tempfile.TemporaryDirectory() as tmp:
        src = os.path.join(tmp, "rhs.cpp")
        exe = os.path.join(tmp, "rhs")
        with open(src, "w") as f:
            f.write(SRC)
        subprocess.run(["g++", "-std=c++17", "-O2", src, "-o", exe], check=True)
        out = []
        for seed, step, corr in CASES:
            txt = subprocess.run([exe, str(seed), str(step), str(corr), str(N)], check=True,
                                 capture_output=True, text=True).stdout.split()
            out.append({"seed": seed, "step": step, "corrector": corr, "values_hex": txt})
    with open(os.path.join(HERE, "seed_seq_rhs.json"), "w") as f:
        json.dump({"n": N, "cases": out}, f)


if __name__ == "__main__":
    main()
