// The checker never evaluates tabulated EOSes; these aliases only let the
// reference translation units instantiate their explicit templates.
#pragma once
#include <grace/physics/eos/piecewise_polytropic_eos.hh>
namespace grace { class tabulated_cold_eos_t : public piecewise_polytropic_eos_t { public: using piecewise_polytropic_eos_t::piecewise_polytropic_eos_t; }; }
