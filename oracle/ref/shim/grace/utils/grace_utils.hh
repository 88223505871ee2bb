// Reduced utility header: only the inline/device/math helpers the per-cell
// numerics need (the full header pulls in MPI/p4est wrappers).
#pragma once
#include <grace_config.h>
#include <grace/utils/inline.h>
#include <grace/utils/device.h>
#include <grace/utils/math.hh>
#include <grace/utils/matrix_helpers.tpp>
#define ERROR(msg) do { throw std::runtime_error("error"); } while (0)
#define ASSERT(c, msg) do { if (!(c)) throw std::runtime_error("assert"); } while (0)
