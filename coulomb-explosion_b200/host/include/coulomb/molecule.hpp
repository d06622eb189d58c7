// molecule.hpp -- atoms, molecules, phase-space state and the unit boundary.
//
// Same data contract as the reference's include/coulomb/molecule.hpp:14-35,
// include/coulomb/units.hpp:11-14 and include/coulomb/system.hpp:13-18: masses
// in electron masses (converted from amu at the input boundary), integer or real
// charges, atomic units with Coulomb constant 1.
#pragma once

#include <string>
#include <utility>
#include <vector>

#include "coulomb/types.hpp"

namespace coulomb {

namespace units {
inline constexpr Real kAmuToElectronMass = 1822.888486209;  // CODATA 2018 m_u / m_e
constexpr Real amu_to_electron_mass(Real mass_amu) { return mass_amu * kAmuToElectronMass; }
}  // namespace units

struct Atom {
  std::string symbol;
  Real mass{0};    // electron masses
  Real charge{0};  // elementary charges
};

inline Atom atom_from_amu(std::string symbol, Real mass_amu, Real charge) {
  return Atom{std::move(symbol), units::amu_to_electron_mass(mass_amu), charge};
}

struct Molecule {
  std::vector<Atom> atoms;
  std::size_t size() const { return atoms.size(); }
  bool empty() const { return atoms.empty(); }
};

struct State {
  std::vector<Vec3> positions;
  std::vector<Vec3> velocities;
  std::size_t size() const { return positions.size(); }
};

// Potential and kinetic energy in double (host-side bookkeeping; the GPU engine
// evaluates its own in-kernel copies).
Real potential_energy(const Molecule& mol, const std::vector<Vec3>& pos, Real coulomb_k = 1.0);
Real kinetic_energy(const Molecule& mol, const std::vector<Vec3>& vel);

// The methane molecule of the reference's dataset generator: C then 4 H, each
// singly ionised (examples/generate_dataset.cpp:56-66).
Molecule make_methane();

}  // namespace coulomb
