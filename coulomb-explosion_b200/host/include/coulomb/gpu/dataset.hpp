// dataset.hpp -- the reference's dataset output format (coulomb::gpu::DatasetWriter).
//
// Fixed-width little-endian records, written field by field with no padding
// (examples/generate_dataset.cpp:10-19, 198-217), readable unchanged by the
// reference's examples/to_parquet.py, examples/verify_subset.py and
// demo/sanity_check.py:
//   n*3 float32  initial positions (atom order as the molecule's symbols)
//   n*3 float32  final momenta m v (after energy redistribution)
//   uint32       accepted steps
//   uint8        converged (1) or not (0)
// plus a JSON sidecar <out>.meta.json with the reference's keys
// (generate_dataset.cpp:118-155) and a few engine keys (device, precision mode,
// sampler, error statistics when known).
#pragma once

#include <cstddef>
#include <cstdint>
#include <fstream>
#include <map>
#include <string>
#include <vector>

#include "coulomb/molecule.hpp"

namespace coulomb::gpu {

inline constexpr std::size_t record_bytes(std::size_t n_atoms) { return n_atoms * 3 * 4 * 2 + 4 + 1; }

class DatasetWriter {
 public:
  DatasetWriter(const std::string& path, const Molecule& mol);
  // Append `count` records; pos / mom are [count][n][3] float, steps [count],
  // converged [count] (non-zero = 1).
  void append(std::size_t count, const float* pos, const float* mom, const std::uint32_t* steps,
              const std::uint8_t* converged);
  std::size_t written() const { return written_; }
  void close();
  // Sidecar JSON. `numbers` are written as JSON numbers, `strings` as strings.
  void write_metadata(const std::map<std::string, double>& numbers,
                      const std::map<std::string, std::string>& strings) const;

 private:
  std::string path_;
  Molecule mol_;
  std::ofstream out_;
  std::vector<char> buf_;
  std::size_t written_ = 0;
};

}  // namespace coulomb::gpu
