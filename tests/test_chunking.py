"""Chunk schedule of the pipelined host-buffer calls (ce_run: chunks of at least
2^16 sims, at most 16; ce_run_mixed: 2^17, at most 8), checked on the CPU: the
chunks cover [0, S) in order with none empty, below 2 minimum chunks there is one,
from 6 chunks on the two at each end weigh 1/4 and 1/2 of a full one, and the
reported largest chunk is the one the device slots are sized for. Also the
default refill granularity and layout per molecule size."""
from __future__ import annotations

import shutil
import subprocess

import pytest

from conftest import ROOT

CSRC = ROOT / "coulomb-explosion_b200" / "csrc"
SIZES = [1, 1000, 131071, 131072, 131073, 196608, 5 * 65536 + 777, 7 * 65536 + 777, 1_000_000, 10_000_000,
         123_456_789, 1 << 40]


@pytest.fixture(scope="module")
def schedule(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path_factory.mktemp("chunk") / "chunk_bounds"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-I", str(ROOT / "include"),
                    "-I", str(CSRC), "-o", str(exe),
                    str(ROOT / "tests" / "cpp" / "chunk_bounds_main.cu")], check=True, capture_output=True)

    def run(min_chunk, max_chunks=None):
        if min_chunk == "stream":
            args = ["stream", *map(str, [1 << 15, 65536, 459529, 1_000_000, 10_000_000, 123_456_789, (1 << 31) - 1])]
        elif max_chunks is None:
            args = [str(min_chunk)]
        else:
            args = [str(min_chunk), str(max_chunks), *map(str, SIZES)]
        out = subprocess.run([str(exe), *args], check=True, capture_output=True, text=True).stdout
        return [list(map(int, line.split())) for line in out.splitlines()]
    return run


@pytest.mark.parametrize("min_chunk,max_chunks", [(1 << 16, 16), (1 << 17, 8)])
def test_chunks_cover_the_batch(schedule, min_chunk, max_chunks):
    for row in schedule(min_chunk, max_chunks):
        S, n, cmax, bnd = row[0], row[1], row[2], row[3:]
        assert len(bnd) == n + 1 and bnd[0] == 0 and bnd[-1] == S
        sizes = [bnd[k + 1] - bnd[k] for k in range(n)]
        assert min(sizes) > 0 and max(sizes) == cmax
        expect = 1 if S < 2 * min_chunk else min(max_chunks, S // min_chunk)
        assert n == expect
        if n >= 6:
            full = sizes[2]
            for k, quarters in ((0, 1), (1, 2), (n - 2, 2), (n - 1, 1)):
                assert abs(sizes[k] - full * quarters / 4) <= 2
        else:
            assert max(sizes) - min(sizes) <= 1


def test_default_refill(schedule):
    # floor((G - 1) / 3) idle groups of G = 32 / n sims per warp, at least one;
    # one thread per sim refills once 4 sims of the warp are idle (a lone atom at once)
    rows = schedule("refill")
    assert [r[0] for r in rows] == list(range(1, 11))
    assert {r[0]: r[1] for r in rows} == {1: 1, 2: 5, 3: 3, 4: 2, 5: 1, 6: 1, 7: 1, 8: 1, 9: 1, 10: 1}
    assert {r[0]: r[2] for r in rows} == {1: 1, **{n: 4 for n in range(2, 11)}}
    # two threads per sim refill once 2 of a warp's 16 sims are idle (at 2 atoms
    # lanes_per_sim = 2 is the lane-per-atom layout)
    assert {r[0]: r[3] for r in rows} == {1: 1, 2: 5, **{n: 2 for n in range(3, 11)}}


def test_default_layout(schedule):
    # lanes_per_sim: 1 = thread per sim, 2 = two threads per sim, n = lane per atom
    rows = {r[0]: r[4:] for r in schedule("refill")}
    fp32 = {n: rows[n][0] for n in rows}
    full = {n: rows[n][1] for n in rows}
    assert fp32 == {1: 1, 2: 1, 3: 1, 4: 1, 5: 1, 6: 1, 7: 2, 8: 2, 9: 2, 10: 2}
    assert full == {1: 1, 2: 2, 3: 3, 4: 1, 5: 1, 6: 1, 7: 7, 8: 2, 9: 9, 10: 2}
    # layout_of(n, 2): 0 thread, 1 two threads, 2 lane per atom
    assert {n: rows[n][2] for n in rows} == {1: 0, 2: 2, **{n: 1 for n in range(3, 11)}}


def test_streamed_chunks(schedule):
    # The streamed ce_run (batches of 2^15 .. 2^31 - 1 sims) cuts the positions
    # into chunks of 2^shift sims: at least 2^14 of them, fewer than 32 chunks,
    # and for any atom count a whole number of 128-byte lines (12 N 2^shift bytes).
    for S, shift, J in schedule("stream"):
        assert shift >= 14 and J == -(-S // (1 << shift)) and J <= 32 and S >> shift < 32, (S, shift, J)
        assert shift == 14 or S >> (shift - 1) >= 32, (S, shift)  # the smallest such chunk
        for n in range(1, 11):
            assert (12 * n << shift) % 128 == 0
    rows = {S: (shift, J) for S, shift, J in schedule("stream")}
    assert rows[1_000_000] == (15, 31) and rows[459529] == (14, 29) and rows[1 << 15] == (14, 2)
