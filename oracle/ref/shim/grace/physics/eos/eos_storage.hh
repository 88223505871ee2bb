// EOS registry stand-in.  The checker constructs EOS objects directly; the
// registry exists only so header-defined parameter helpers compile.
#pragma once
#include <grace/physics/eos/eos_base.hh>
#include <grace/physics/eos/hybrid_eos.hh>
#include <grace/physics/eos/piecewise_polytropic_eos.hh>
#include <grace/physics/eos/tabulated_cold_eos.hh>
#include <grace/physics/eos/ideal_gas_eos.hh>
#include <grace/physics/eos/tabulated_eos.hh>
#include <stdexcept>
namespace grace {
struct eos {
  static eos& get() { static eos e; return e; }
  template <class T> T& get_eos() { throw std::runtime_error("eos registry not available in checker"); }
};
}
