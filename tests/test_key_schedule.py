"""CPU test of the Philox round-key schedule that the move kernels take as a
launch parameter: a Philox4x32-10 evaluated with the precomputed keys of
`philox_schedule` (both words, or only the second with the first advanced in
place) gives the oracle's words for every counter, so the keyed kernel
instances draw the same numbers as the ones that advance the key themselves.
The schedule is compiled from the library's own header."""
import os
import subprocess

import numpy as np

from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <cstdio>
#include <cstdint>
#include "scmf_internal.h"
using namespace scmf;
static void round_(uint32_t c[4], uint32_t k0, uint32_t k1) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0], p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0, n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
    c[0] = n0; c[1] = (uint32_t)p1; c[2] = n2; c[3] = (uint32_t)p0;
}
int main() {
    unsigned k0, k1, x, y, z, w;
    while (std::scanf("%u %u %u %u %u %u", &k0, &k1, &x, &y, &z, &w) == 6) {
        const PhiloxKeys ks = philox_schedule(k0, k1);
        uint32_t a[4] = {x, y, z, w}, b[4] = {x, y, z, w};
        uint32_t kk0 = k0;
        for (int r = 0; r < 10; ++r) {
            round_(a, ks.k[2 * r], ks.k[2 * r + 1]);   // both words from the schedule
            round_(b, kk0, ks.k[2 * r + 1]);           // first word advanced in place
            kk0 += 0x9E3779B9u;
        }
        std::printf("%u %u %u %u %u %u %u %u\n", a[0], a[1], a[2], a[3], b[0], b[1], b[2], b[3]);
    }
    return 0;
}
"""


def test_round_key_schedule_matches_oracle(tmp_path):
    src = tmp_path / "ks.cpp"
    exe = tmp_path / "ks"
    src.write_text(PROGRAM)
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I",
                    os.path.join(ROOT, "new_arch_b200", "csrc"), str(src), "-o", str(exe)], check=True)
    rng = np.random.default_rng(3)
    rows = rng.integers(0, 2**32, size=(200, 6), dtype=np.uint64)
    rows[:4, :2] = [[0, 0], [0xFFFFFFFF, 0xFFFFFFFF], [7, 0], [1000, 0]]
    text = "\n".join(" ".join(str(int(v)) for v in r) for r in rows) + "\n"
    out = subprocess.run([str(exe)], input=text, capture_output=True, text=True, check=True).stdout.split("\n")
    for r, line in zip(rows, out):
        got = np.array([int(v) for v in line.split()], dtype=np.uint32)
        want = orc.philox(r[2:6].astype(np.uint32), r[:2].astype(np.uint32))
        assert np.array_equal(got[:4], want), r
        assert np.array_equal(got[4:], want), r
