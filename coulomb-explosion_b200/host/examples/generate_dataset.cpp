// generate_dataset.cpp -- Coulomb-explosion dataset generator on the B200 engine.
//
// Drop-in for the reference's examples/generate_dataset.cpp, built beside the
// reference's coulomb::engine (its Molecule and UniformSphereSampler): same flags and
// defaults (--out --sims --seed --radius --min-separation --rtol --atol
// --pe-stop --progress-every; CH4 singly ionised, 1e7 sims, seed 49188291,
// r 4.0, min_sep 0.25, rtol 1e-4, atol 1e-7, pe_stop 1e-5), same record format
// and sidecar (coulomb/gpu/dataset.hpp), readable by the reference's to_parquet.py,
// verify_subset.py and sanity_check.py. Added flags:
//   --sampler uniform-sphere|philox   the reference's sequential mt19937_64
//        sampler on the host (bit-identical geometries to the reference run with
//        the same seed), or the counter-based sampler on the device (default)
//   --chunk N                         sims per device chunk (default 1e6)
//   --precision-mode 0..3             CE_PREC_* bits (default 3)
//   --device D
// Pipeline per chunk: sample (device or host) -> integrate on the compute
// stream -> copy positions / momenta / steps / status into pinned host buffers
// on a copy stream -> the host writes chunk c-1 while chunk c integrates.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "ce_gpu.h"
#include "ce_sampler.h"
#include "coulomb/gpu/dataset.hpp"
#include "coulomb/molecule.hpp"
#include "coulomb/sampler.hpp"
#include "coulomb/system.hpp"

using namespace coulomb;
using gpu::DatasetWriter;
using Clock = std::chrono::steady_clock;

namespace {

// Methane, singly ionised on every atom: C then 4 H (the reference generator's
// molecule, examples/generate_dataset.cpp:56-66).
Molecule make_methane() {
  Molecule m;
  m.atoms.push_back(atom_from_amu("C", static_cast<Real>(12.011), Real{1}));
  for (int i = 0; i < 4; ++i) m.atoms.push_back(atom_from_amu("H", static_cast<Real>(1.008), Real{1}));
  return m;
}

struct Args {
  std::size_t sims = 10'000'000;
  std::uint64_t seed = 49188291;
  double radius = 4.0;
  double min_separation = 0.25;
  double rtol = 1e-4;
  double atol = 1e-7;
  double pe_stop = 1e-5;
  std::string out;
  std::size_t progress_every = 2000;
  std::string sampler = "philox";
  std::size_t chunk = 1'000'000;
  int precision_mode = 3;
  int device = 0;
};

[[noreturn]] void usage(const std::string& bad) {
  std::fprintf(stderr, "unknown or incomplete argument: %s\n", bad.c_str());
  std::exit(EXIT_FAILURE);
}

Args parse(int argc, char** argv) {
  Args a;
  for (int i = 1; i < argc; ++i) {
    const std::string f = argv[i];
    if (i + 1 >= argc) usage(f);
    const std::string v = argv[++i];
    if (f == "--sims") a.sims = std::stoull(v);
    else if (f == "--seed") a.seed = std::stoull(v);
    else if (f == "--radius") a.radius = std::stod(v);
    else if (f == "--min-separation") a.min_separation = std::stod(v);
    else if (f == "--rtol") a.rtol = std::stod(v);
    else if (f == "--atol") a.atol = std::stod(v);
    else if (f == "--pe-stop") a.pe_stop = std::stod(v);
    else if (f == "--out") a.out = v;
    else if (f == "--progress-every") a.progress_every = std::stoull(v);
    else if (f == "--sampler") a.sampler = v;
    else if (f == "--chunk") a.chunk = std::stoull(v);
    else if (f == "--precision-mode") a.precision_mode = std::stoi(v);
    else if (f == "--device") a.device = std::stoi(v);
    else usage(f);
  }
  if (a.out.empty()) {
    std::fprintf(stderr, "--out is required\n");
    std::exit(EXIT_FAILURE);
  }
  if (a.sampler != "philox" && a.sampler != "uniform-sphere") usage("--sampler " + a.sampler);
  if (a.chunk == 0) usage("--chunk 0");
  return a;
}

void check(cudaError_t st, const char* what) {
  if (st != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(st));
}

struct Slot {
  float* d_pos = nullptr;
  float* d_mom = nullptr;
  uint32_t* d_steps = nullptr;
  uint8_t* d_status = nullptr;
  float* h_pos = nullptr;
  float* h_mom = nullptr;
  uint32_t* h_steps = nullptr;
  uint8_t* h_status = nullptr;
  cudaEvent_t copied = nullptr;
  std::size_t count = 0;
};

}  // namespace

int main(int argc, char** argv) {
  try {
    const Args args = parse(argc, argv);
    const Molecule mol = make_methane();
    const std::size_t n = mol.size(), n3 = n * 3;
    std::printf("CH4 dataset generator (B200): n_sims=%zu chunk=%zu sampler=%s rtol=%.0e atol=%.0e pe_stop=%.0e\n",
                args.sims, args.chunk, args.sampler.c_str(), args.rtol, args.atol, args.pe_stop);

    ce_engine* e = nullptr;
    if (ce_create(&e, args.device) != CE_OK) throw std::runtime_error("no usable B200");
    std::vector<double> m(n), q(n);
    for (std::size_t i = 0; i < n; ++i) {
      m[i] = static_cast<double>(mol.atoms[i].mass);
      q[i] = static_cast<double>(mol.atoms[i].charge);
    }
    if (ce_set_molecule(e, static_cast<int>(n), m.data(), q.data(), 1.0) != CE_OK)
      throw std::runtime_error(ce_last_error(e));
    ce_run_config cfg;
    ce_default_config(&cfg);
    cfg.rtol = args.rtol;
    cfg.atol = args.atol;
    cfg.pe_stop_fraction = args.pe_stop;
    cfg.precision_mode = args.precision_mode;

    cudaStream_t compute, copy;
    check(cudaStreamCreateWithFlags(&compute, cudaStreamNonBlocking), "stream");
    check(cudaStreamCreateWithFlags(&copy, cudaStreamNonBlocking), "stream");
    const std::size_t C = std::min(args.chunk, std::max<std::size_t>(args.sims, 1));
    Slot slots[2];
    for (Slot& s : slots) {
      check(cudaMalloc(&s.d_pos, C * n3 * sizeof(float)), "cudaMalloc");
      check(cudaMalloc(&s.d_mom, C * n3 * sizeof(float)), "cudaMalloc");
      check(cudaMalloc(&s.d_steps, C * sizeof(uint32_t)), "cudaMalloc");
      check(cudaMalloc(&s.d_status, C), "cudaMalloc");
      check(cudaMallocHost(&s.h_pos, C * n3 * sizeof(float)), "cudaMallocHost");
      check(cudaMallocHost(&s.h_mom, C * n3 * sizeof(float)), "cudaMallocHost");
      check(cudaMallocHost(&s.h_steps, C * sizeof(uint32_t)), "cudaMallocHost");
      check(cudaMallocHost(&s.h_status, C), "cudaMallocHost");
      check(cudaEventCreateWithFlags(&s.copied, cudaEventDisableTiming), "event");
    }
    cudaEvent_t integrated;
    check(cudaEventCreateWithFlags(&integrated, cudaEventDisableTiming), "event");

    UniformSphereSampler host_sampler({static_cast<Real>(args.radius), static_cast<Real>(args.min_separation), 10000},
                                      args.seed);
    const ce_ball_sampler dev_sampler{args.seed, args.radius, args.min_separation, 0};
    DatasetWriter writer(args.out, mol);
    std::size_t n_failed = 0, done = 0, steps_sum = 0;
    const auto t0 = Clock::now();

    auto flush_slot = [&](Slot& s) {
      check(cudaEventSynchronize(s.copied), "cudaEventSynchronize");
      std::vector<uint8_t> conv(s.count);
      for (std::size_t k = 0; k < s.count; ++k) {
        conv[k] = s.h_status[k] == CE_SIM_OK ? 1 : 0;
        n_failed += conv[k] ? 0 : 1;
        steps_sum += s.h_steps[k];
      }
      writer.append(s.count, s.h_pos, s.h_mom, s.h_steps, conv.data());
      done += s.count;
      s.count = 0;
    };

    std::size_t chunk_id = 0;
    for (std::size_t first = 0; first < args.sims; first += C, ++chunk_id) {
      Slot& s = slots[chunk_id % 2];
      if (s.count) flush_slot(s);  // this slot's previous chunk must be on disk first
      const std::size_t cnt = std::min(C, args.sims - first);
      if (args.sampler == "philox") {
        if (ce_sample_ball_device(static_cast<int>(n), first, cnt, &dev_sampler, s.d_pos, nullptr, compute) != CE_OK)
          throw std::runtime_error("ce_sample_ball_device failed");
      } else {
        State st;
        for (std::size_t k = 0; k < cnt; ++k) {
          host_sampler.sample(mol, st);
          for (std::size_t i = 0; i < n; ++i) {
            s.h_pos[k * n3 + i * 3 + 0] = static_cast<float>(st.positions[i].x);
            s.h_pos[k * n3 + i * 3 + 1] = static_cast<float>(st.positions[i].y);
            s.h_pos[k * n3 + i * 3 + 2] = static_cast<float>(st.positions[i].z);
          }
        }
        check(cudaMemcpyAsync(s.d_pos, s.h_pos, cnt * n3 * sizeof(float), cudaMemcpyHostToDevice, compute), "H2D");
      }
      ce_outputs out{s.d_mom, nullptr, s.d_steps, s.d_status, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
      if (ce_run_device(e, cnt, s.d_pos, &cfg, &out, compute) != CE_OK) throw std::runtime_error(ce_last_error(e));
      check(cudaEventRecord(integrated, compute), "event");
      check(cudaStreamWaitEvent(copy, integrated, 0), "wait");
      if (args.sampler == "philox")
        check(cudaMemcpyAsync(s.h_pos, s.d_pos, cnt * n3 * sizeof(float), cudaMemcpyDeviceToHost, copy), "D2H");
      check(cudaMemcpyAsync(s.h_mom, s.d_mom, cnt * n3 * sizeof(float), cudaMemcpyDeviceToHost, copy), "D2H");
      check(cudaMemcpyAsync(s.h_steps, s.d_steps, cnt * sizeof(uint32_t), cudaMemcpyDeviceToHost, copy), "D2H");
      check(cudaMemcpyAsync(s.h_status, s.d_status, cnt, cudaMemcpyDeviceToHost, copy), "D2H");
      check(cudaEventRecord(s.copied, copy), "event");
      s.count = cnt;
      Slot& other = slots[(chunk_id + 1) % 2];
      if (other.count) flush_slot(other);  // overlaps this chunk's integration
      if (args.progress_every && (chunk_id + 1) % std::max<std::size_t>(1, args.progress_every / 1000) == 0) {
        const double el = std::chrono::duration<double>(Clock::now() - t0).count();
        std::fprintf(stderr, "\r%zu/%zu sims (%.0f sims/sec)   ", done, args.sims, done / std::max(el, 1e-9));
      }
    }
    for (Slot& s : slots)
      if (s.count) flush_slot(s);
    writer.close();
    const double wall = std::chrono::duration<double>(Clock::now() - t0).count();
    std::fprintf(stderr, "\n");
    std::printf("done: %zu sims in %.2fs (%.0f sims/sec), %zu failed to converge\n", done, wall, done / wall, n_failed);
    writer.write_metadata({{"n_sims", static_cast<double>(args.sims)},
                           {"seed", static_cast<double>(args.seed)},
                           {"radius", args.radius},
                           {"min_separation", args.min_separation},
                           {"rtol", args.rtol},
                           {"atol", args.atol},
                           {"pe_stop", args.pe_stop},
                           {"lanes", static_cast<double>(C)},
                           {"n_failed_convergence", static_cast<double>(n_failed)},
                           {"wall_seconds", wall},
                           {"sims_per_sec", done / wall},
                           {"mean_steps", done ? static_cast<double>(steps_sum) / done : 0.0},
                           {"precision_mode", static_cast<double>(args.precision_mode)}},
                          {{"sampler", args.sampler}, {"engine", ce_version()}});
    std::printf("wrote %s and %s.meta.json\n", args.out.c_str(), args.out.c_str());
    for (Slot& s : slots) {
      cudaFree(s.d_pos);
      cudaFree(s.d_mom);
      cudaFree(s.d_steps);
      cudaFree(s.d_status);
      cudaFreeHost(s.h_pos);
      cudaFreeHost(s.h_mom);
      cudaFreeHost(s.h_steps);
      cudaFreeHost(s.h_status);
      cudaEventDestroy(s.copied);
    }
    cudaEventDestroy(integrated);
    cudaStreamDestroy(compute);
    cudaStreamDestroy(copy);
    ce_destroy(e);
    return EXIT_SUCCESS;
  } catch (const std::exception& ex) {
    std::fprintf(stderr, "error: %s\n", ex.what());
    return EXIT_FAILURE;
  }
}
