#pragma once
#include <Kokkos_Core.hpp>
namespace grace { using default_space = Kokkos::HostSpace; }
