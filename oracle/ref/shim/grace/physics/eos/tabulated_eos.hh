#pragma once
#include <grace/physics/eos/hybrid_eos.hh>
#include <grace/physics/eos/piecewise_polytropic_eos.hh>
namespace grace { class tabulated_eos_t : public hybrid_eos_t<piecewise_polytropic_eos_t> { public: using hybrid_eos_t<piecewise_polytropic_eos_t>::hybrid_eos_t; }; }
