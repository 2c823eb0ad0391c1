"""CPU check of the tensor-core GEMM's shared-memory contract (no GPU).

The GEMM (csrc/mlp.cu) stages operand tiles with tc::tile_offset and points
each tcgen05.mma at them with tc::smem_desc. This test compiles a small host
program against csrc/tcgen05.cuh, decodes the descriptors it produces, and
walks the K-major, no-swizzle canonical operand layout the hardware reads
(8 rows of 16 bytes per core matrix; the two 8-element K chunks of one MMA
LBO bytes apart; 8-row groups SBO bytes apart) to require that every element
an MMA reads is the element the staging code stored there. It also checks the
instruction descriptor's fields.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "sovereign-solver_b200", "csrc")

HARNESS = r"""
#include <cstdio>
#include "tcgen05.cuh"
int main() {
    using namespace pdhg::tc;
    const unsigned base = 0x2400;  // a 1024-aligned shared-memory address
    for (int s = 0; s < kTileK / 16; ++s)
        std::printf("desc %d %llu\n", s, (unsigned long long)smem_desc(base + s * 2 * kChunkBytes));
    for (int r = 0; r < kTileM; ++r)
        for (int k = 0; k < kTileK; ++k) std::printf("off %d %d %d\n", r, k, tile_offset(r, k));
    std::printf("idesc %u\n", instr_desc_bf16(128));
    std::printf("base %u\n", base);
    return 0;
}
"""


@pytest.fixture(scope="module")
def harness_output(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    d = tmp_path_factory.mktemp("tc")
    src = d / "h.cu"
    src.write_text(HARNESS)
    exe = d / "h"
    subprocess.run([nvcc, "-std=c++17", "-I", CSRC, str(src), "-o", str(exe)], check=True,
                   capture_output=True, timeout=300)
    return subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout


def parse(out):
    desc, off = {}, {}
    idesc = base = None
    for line in out.splitlines():
        f = line.split()
        if f[0] == "desc":
            desc[int(f[1])] = int(f[2])
        elif f[0] == "off":
            off[(int(f[1]), int(f[2]))] = int(f[3])
        elif f[0] == "idesc":
            idesc = int(f[1])
        elif f[0] == "base":
            base = int(f[1])
    return desc, off, idesc, base


def test_every_mma_reads_the_staged_element(harness_output):
    desc, off, _, base = parse(harness_output)
    # staging: each (row, k) has its own 2-byte slot inside the 16 KB tile
    assert sorted(off.values()) == list(range(128 * 64))
    for s, d in desc.items():
        start = (d & 0x3FFF) << 4
        lbo = ((d >> 16) & 0x3FFF) << 4
        sbo = ((d >> 32) & 0x3FFF) << 4
        assert (d >> 46) & 0x3 == 1          # descriptor version of sm_100
        assert (d >> 61) & 0x7 == 0          # no swizzle
        assert (d >> 49) & 0x7 == 0          # base offset
        for r in range(128):
            for kk in range(16):
                hw = start + (r % 8) * 16 + (r // 8) * sbo + (kk // 8) * lbo + (kk % 8) * 2
                assert hw == base + 2 * off[(r, 16 * s + kk)], (s, r, kk)


def test_instruction_descriptor_fields(harness_output):
    _, _, idesc, _ = parse(harness_output)
    assert (idesc >> 4) & 0x3 == 1        # accumulator FP32
    assert (idesc >> 7) & 0x7 == 1        # A BF16
    assert (idesc >> 10) & 0x7 == 1       # B BF16
    assert (idesc >> 15) & 0x1 == 0       # A K-major
    assert (idesc >> 16) & 0x1 == 0       # B K-major
    assert ((idesc >> 17) & 0x3F) << 3 == 128   # N
    assert ((idesc >> 24) & 0x1F) << 4 == 128   # M
    assert idesc & 0x7 == 0 and (idesc >> 13) & 0x3 == 0   # dense, no negation
