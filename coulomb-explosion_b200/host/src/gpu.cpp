// gpu.cpp -- coulomb::gpu::Engine, BatchedRK45 and run_to_convergence_batch:
// the reference's batched and scalar drivers over the C ABI of libce_gpu.so,
// taking and returning the reference's own coulomb:: types.
#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>

#include "ce_gpu.h"
#include "coulomb/gpu/batched_rk45.hpp"

namespace coulomb::gpu {

Engine::Engine(int device) {
  const int rc = ce_create(&e_, device);
  if (rc == CE_ERR_INVALID) throw std::invalid_argument("coulomb::gpu::Engine: bad device index");
  if (rc != CE_OK) throw std::runtime_error("coulomb::gpu::Engine: no usable B200 (ce_create " + std::to_string(rc) + ")");
}

Engine::~Engine() { ce_destroy(e_); }

void Engine::throw_last(int rc, const char* what) const {
  const std::string msg = std::string(what) + ": " + ce_last_error(e_);
  if (rc == CE_ERR_INVALID || rc == CE_ERR_STATE) throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

void Engine::set_molecule(const Molecule& mol, Real coulomb_k) {
  std::vector<double> m(mol.size()), q(mol.size());
  for (std::size_t i = 0; i < mol.size(); ++i) {
    m[i] = static_cast<double>(mol.atoms[i].mass);
    q[i] = static_cast<double>(mol.atoms[i].charge);
  }
  const int rc = ce_set_molecule(e_, static_cast<int>(mol.size()), m.data(), q.data(), static_cast<double>(coulomb_k));
  if (rc != CE_OK) throw_last(rc, "ce_set_molecule");
}

namespace {

ce_run_config to_c(const RunConfig& cfg, double rtol, double atol, int mode) {
  ce_run_config c;
  ce_default_config(&c);
  c.rtol = rtol;
  c.atol = atol;
  c.pe_stop_fraction = static_cast<double>(cfg.pe_stop_fraction);
  c.max_dt = static_cast<double>(cfg.max_dt);
  c.max_steps = cfg.max_steps;
  c.redistribute_energy = cfg.redistribute_energy ? 1 : 0;
  c.precision_mode = mode;
  return c;
}

}  // namespace

BatchedRK45::BatchedRK45(const Molecule& mol, Real coulomb_k, std::size_t lanes, Real rtol, Real atol, int device,
                         int precision_mode)
    : n_(mol.size()), lanes_(lanes), rtol_(rtol), atol_(atol), mode_(precision_mode) {
  if (lanes == 0) throw std::invalid_argument("BatchedRK45: lanes must be positive");
  engine_ = std::make_unique<Engine>(device);
  engine_->set_molecule(mol, coulomb_k);
  pos_.assign(lanes * n_ * 3, 0.0f);
}

BatchedRK45::~BatchedRK45() = default;

void BatchedRK45::set_lane_geometry(std::size_t lane, const std::vector<Vec3>& pos) {
  if (lane >= lanes_) throw std::invalid_argument("BatchedRK45: lane out of range");
  if (pos.size() != n_) throw std::invalid_argument("BatchedRK45: geometry has the wrong atom count");
  for (std::size_t i = 0; i < n_; ++i) {
    pos_[(lane * n_ + i) * 3 + 0] = static_cast<float>(pos[i].x);
    pos_[(lane * n_ + i) * 3 + 1] = static_cast<float>(pos[i].y);
    pos_[(lane * n_ + i) * 3 + 2] = static_cast<float>(pos[i].z);
  }
}

BatchedRK45::Result BatchedRK45::run(const RunConfig& cfg) {
  const ce_run_config c = to_c(cfg, rtol_, atol_, mode_);
  std::vector<float> mom(lanes_ * n_ * 3);
  std::vector<std::uint32_t> steps(lanes_), rejects(lanes_);
  std::vector<std::uint8_t> status(lanes_);
  Result r;
  r.ker.resize(lanes_);
  ce_outputs out{mom.data(), r.ker.data(), steps.data(), status.data(), rejects.data(), nullptr, nullptr, nullptr,
                 nullptr, nullptr};
  const int rc = ce_run(engine_->handle(), lanes_, pos_.data(), &c, &out);
  if (rc != CE_OK) engine_->throw_last(rc, "ce_run");
  r.momenta.assign(mom.begin(), mom.end());
  r.steps.assign(steps.begin(), steps.end());
  r.rejects = rejects;
  r.converged.resize(lanes_);
  r.status.resize(lanes_);
  for (std::size_t l = 0; l < lanes_; ++l) {
    r.status[l] = static_cast<SimStatus>(status[l]);
    r.converged[l] = status[l] == CE_SIM_OK ? 1 : 0;
    r.batch_steps = std::max<std::size_t>(r.batch_steps, steps[l]);
  }
  return r;
}

std::vector<RunResult> run_to_convergence_batch(const Molecule& mol, std::vector<State>& states, const RunConfig& cfg,
                                                const IntegratorOptions& opts, Real coulomb_k, int device,
                                                int precision_mode, BatchStatus* extra) {
  const std::size_t S = states.size(), n = mol.size();
  std::vector<RunResult> res(S);
  if (S == 0) return res;
  Engine eng(device);
  eng.set_molecule(mol, coulomb_k);
  std::vector<float> pos(S * n * 3), mom(S * n * 3);
  for (std::size_t s = 0; s < S; ++s) {
    if (states[s].size() != n) throw std::invalid_argument("run_to_convergence_batch: state size mismatch");
    for (const Vec3& v : states[s].velocities)
      if (v.x != 0 || v.y != 0 || v.z != 0)
        throw std::invalid_argument("run_to_convergence_batch: every simulation must start at rest");
    for (std::size_t i = 0; i < n; ++i) {
      pos[(s * n + i) * 3 + 0] = static_cast<float>(states[s].positions[i].x);
      pos[(s * n + i) * 3 + 1] = static_cast<float>(states[s].positions[i].y);
      pos[(s * n + i) * 3 + 2] = static_cast<float>(states[s].positions[i].z);
    }
  }
  std::vector<double> ker(S), t_final(S), pe_final(S), ke_before(S), e0(S);
  std::vector<std::uint32_t> steps(S), rejects(S);
  std::vector<std::uint8_t> status(S);
  ce_outputs out{mom.data(), ker.data(), steps.data(), status.data(), rejects.data(), t_final.data(),
                 pe_final.data(), ke_before.data(), nullptr, e0.data()};
  const ce_run_config c = to_c(cfg, static_cast<double>(opts.rtol), static_cast<double>(opts.atol), precision_mode);
  const int rc = ce_run(eng.handle(), S, pos.data(), &c, &out);
  if (rc != CE_OK) eng.throw_last(rc, "ce_run");
  if (extra) {
    extra->status.resize(S);
    extra->rejects = rejects;
  }
  for (std::size_t s = 0; s < S; ++s) {
    // energy_initial is E0 = PE0 of the geometry the device integrated (narrowed
    // to float like BatchedRK45<float>::set_lane_geometry), the energy the
    // redistribution restores.
    RunResult& r = res[s];
    r.steps = steps[s];
    r.t_final = static_cast<Real>(t_final[s]);
    r.energy_initial = static_cast<Real>(e0[s]);
    r.pe_final = static_cast<Real>(pe_final[s]);
    r.ke_before_redist = static_cast<Real>(ke_before[s]);
    r.ke_after_redist = static_cast<Real>(ker[s]);
    r.redistribution_scale = static_cast<Real>(
        (cfg.redistribute_energy && ke_before[s] > 0) ? std::sqrt(e0[s] / ke_before[s]) : 1.0);
    r.converged = status[s] == CE_SIM_OK;
    if (extra) extra->status[s] = static_cast<SimStatus>(status[s]);
    for (std::size_t i = 0; i < n; ++i) {
      const double m = static_cast<double>(mol.atoms[i].mass);
      states[s].velocities[i] = Vec3{static_cast<Real>(mom[(s * n + i) * 3] / m),
                                     static_cast<Real>(mom[(s * n + i) * 3 + 1] / m),
                                     static_cast<Real>(mom[(s * n + i) * 3 + 2] / m)};
    }
  }
  return res;
}

}  // namespace coulomb::gpu
