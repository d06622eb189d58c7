// Prints the chunk schedule of the pipelined host-buffer paths (ce::chunk_bounds)
// (with the first argument "stream", the streamed ce_run's chunking instead)
// for the sizes given on the command line: "S nchunks cmax b0 b1 ... bn" per line;
// with the single argument "refill", per atom count n = 1..10 the default refill
// granularity (ce::default_refill) of the lane-per-atom, thread-per-sim and
// two-thread layouts, the default layout (ce::default_lanes) in plain FP32 and in
// the full precision form, and the layout lanes_per_sim = 2 selects
// (ce::layout_of): "n lane thread pair lanes_fp32 lanes_full layout_of_2".
// Host code only; compiled by tests/test_chunking.py.
#include <cstdio>
#include <cstdlib>

#include "engine.hpp"

int main(int argc, char** argv) {
  if (argc >= 2 && argv[1][0] == 's') {  // "stream S...": S, the streamed chunk shift and chunk count
    for (int a = 2; a < argc; ++a) {
      const uint64_t S = std::strtoull(argv[a], nullptr, 10);
      const unsigned sh = ce::io_chunk_shift(S);
      std::printf("%llu %u %llu\n", static_cast<unsigned long long>(S), sh,
                  static_cast<unsigned long long>((S + (1ull << sh) - 1) >> sh));
    }
    return 0;
  }
  if (argc == 2 && argv[1][0] == 'r') {
    for (int n = 1; n <= 10; ++n)
      std::printf("%d %d %d %d %d %d %d\n", n, ce::default_refill(n, n), ce::default_refill(n, 1),
                  ce::default_refill(n, 2), ce::default_lanes(n, 0), ce::default_lanes(n, 3), ce::layout_of(n, 2));
    return 0;
  }
  for (int a = 3; a < argc; ++a) {
    const uint64_t S = std::strtoull(argv[a], nullptr, 10);
    uint64_t bnd[17], cmax = 0;
    const uint64_t n = ce::chunk_bounds(S, std::strtoull(argv[1], nullptr, 10), std::strtoull(argv[2], nullptr, 10),
                                        bnd, &cmax);
    std::printf("%llu %llu %llu", static_cast<unsigned long long>(S), static_cast<unsigned long long>(n),
                static_cast<unsigned long long>(cmax));
    for (uint64_t k = 0; k <= n; ++k) std::printf(" %llu", static_cast<unsigned long long>(bnd[k]));
    std::printf("\n");
  }
  return 0;
}
